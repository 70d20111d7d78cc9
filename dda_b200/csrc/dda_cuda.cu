// dda_cuda.cu -- host side of libdda_b200.so: the C ABI of include/dda_cuda.h.
//
// A context owns the device-resident problem (geometry tables, FFT plans,
// the D-matrix octant in FP64 and/or FP32), the matvec work buffers and the
// Krylov vectors and scalar state for up to max_rhs right-hand sides.  Solves
// run entirely on the device: scalars never leave it during the iteration
// (compare the host round trips of DDA/GpuQmrCs.cpp:146-177); the host only
// polls the per-rhs `done` flags between batches of iterations, which are
// replayed from a captured CUDA graph.

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <array>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dda_cuda.h"
#include "../../include/dda_frontend.h"
#include "dmatrix_kernels.cuh"
#include "farfield_kernels.cuh"
#include "fft_engine.cuh"
#include "kernel_shapes.cuh"
#include "krylov_kernels.cuh"
#include "krylov_ops.cuh"
#include "matvec_kernels.cuh"
#include "matvec_dispatch.cuh"
#include "matvec_planned.cuh"
#include "reduce.cuh"

using namespace dda;

namespace {

thread_local std::string g_create_error;

struct DdaError : std::runtime_error {
  int code;
  DdaError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      throw DdaError(e_ == cudaErrorMemoryAllocation ? DDA_ERR_OOM : DDA_ERR_CUDA,        \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                 \
  } while (0)

// Kernel shapes (threads per CTA): kNtX, NtYz, kNtC in kernel_shapes.cuh.
#define kNtYz NtYz<T>::v
constexpr int kNtV = 256;                 // k_vec
constexpr int kVecPartsMax = 8 * 148;     // k_vec CTAs per right-hand side, at most
constexpr size_t kSmemMax = 227 * 1024;

// Opts kernel f into the whole shared memory of an SM (less its static
// shared memory).  The limit is a
// process-wide attribute of the function, shared by every context (and
// thread) that launches it, so it is always set to the same maximum; each
// launch's own size is checked against kSmemMax by its caller.
// A named range on the host timeline (NVTX) for Nsight Systems: context
// set-up, D matrix, autotuning, solves and their rounds, refinement, far
// field.  Free when no tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

inline cudaError_t allow_smem(const void* f) {
  cudaFuncAttributes a;
  cudaError_t rc = cudaFuncGetAttributes(&a, f);
  if (rc != cudaSuccess) return rc;
  const size_t room = kSmemMax > a.sharedSizeBytes ? kSmemMax - a.sharedSizeBytes : 0;  // minus static
  return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)room);
}

// Device allocations that a context keeps go through dmalloc, which counts
// them for the thread building the context (dda_matvec_layout reports the
// total of dda_create); temporaries use cudaMalloc directly.
// Allocations are stream ordered (cudaMallocAsync / cudaFreeAsync on the
// context stream), so creating or destroying a context never waits for the
// work of other contexts on the device.
thread_local size_t g_dalloc_bytes = 0;
thread_local cudaStream_t g_alloc_stream = nullptr;

void dmalloc(void** p, size_t bytes) {
  CK(cudaMallocAsync(p, bytes, g_alloc_stream));
  g_dalloc_bytes += bytes;
}

// ----------------------------------------------------------- FFT plans ----
struct FftPlan {
  int n = 0;
  std::vector<int> radix;
  std::vector<int> pos_h;  // frequency -> position after a forward transform
  float2* tw32 = nullptr;
  double2* tw64 = nullptr;
  int* freq = nullptr;     // device: position -> frequency
  int* pos = nullptr;      // device: frequency -> position

  // radices: a compile-time plan's stage radices, or empty for the runtime
  // engine's factorisation (8s, then 4, 2, 3, 5, 7).
  void create(int n_, const std::vector<int>& radices = {}) {
    n = n_;
    int m = n;
    if (!radices.empty()) {
      radix = radices;
      for (int r : radix) m /= r;
    } else {
      while (m % 8 == 0) { radix.push_back(8); m /= 8; }
      while (m % 4 == 0) { radix.push_back(4); m /= 4; }
      while (m % 2 == 0) { radix.push_back(2); m /= 2; }
      while (m % 3 == 0) { radix.push_back(3); m /= 3; }
      while (m % 5 == 0) { radix.push_back(5); m /= 5; }
      while (m % 7 == 0) { radix.push_back(7); m /= 7; }
    }
    if (m != 1) throw DdaError(DDA_ERR_UNSUPPORTED, "FFT length " + std::to_string(n) + " is not 2,3,5,7-smooth");
    if ((int)radix.size() > 8) throw DdaError(DDA_ERR_UNSUPPORTED, "FFT length too large");
    std::vector<double2> h64(n);
    std::vector<float2> h32(n);
    const long double two_pi = 6.2831853071795864769252867665590056L;
    for (int k = 0; k < n; k++) {
      long double a = -two_pi * (long double)k / (long double)n;
      long double c = cosl(a), s = sinl(a);
      h64[k] = make_double2((double)c, (double)s);
      h32[k] = make_float2((float)c, (float)s);
    }
    dmalloc((void**)&tw64, n * sizeof(double2));
    dmalloc((void**)&tw32, n * sizeof(float2));
    CK(cudaMemcpyAsync(tw64, h64.data(), n * sizeof(double2), cudaMemcpyHostToDevice, g_alloc_stream));
    CK(cudaMemcpyAsync(tw32, h32.data(), n * sizeof(float2), cudaMemcpyHostToDevice, g_alloc_stream));
    // Mixed-radix digit reversal of the decimation-in-frequency transform:
    // frequency k = d0 + R0 d1 + R0 R1 d2 + ... sits at position
    // d0 n/R0 + d1 n/(R0 R1) + ...
    pos_h.assign(n, 0);
    std::vector<int> fr(n);
    for (int k = 0; k < n; k++) {
      int p = 0, rem = k, unit = n;
      for (int R : radix) {
        unit /= R;
        p += (rem % R) * unit;
        rem /= R;
      }
      pos_h[k] = p;
      fr[p] = k;
    }
    dmalloc((void**)&freq, n * sizeof(int));
    dmalloc((void**)&pos, n * sizeof(int));
    CK(cudaMemcpyAsync(freq, fr.data(), n * sizeof(int), cudaMemcpyHostToDevice, g_alloc_stream));
    CK(cudaMemcpyAsync(pos, pos_h.data(), n * sizeof(int), cudaMemcpyHostToDevice, g_alloc_stream));
  }
  template <typename T> FftPlanDev dev() const {
    FftPlanDev d;
    memset(&d, 0, sizeof(d));
    d.n = n;
    d.nst = (int)radix.size();
    d.packed = 0;  // runtime-engine radices (< 16); unused by planned kernels
    for (size_t i = 0; i < radix.size(); i++) d.packed |= (uint32_t)(radix[i] & 15) << (4 * i);
    d.tw = std::is_same<T, float>::value ? (const void*)tw32 : (const void*)tw64;
    d.freq = freq;
    return d;
  }
  void release(cudaStream_t s) {
    if (tw32) cudaFreeAsync(tw32, s);
    if (tw64) cudaFreeAsync(tw64, s);
    if (freq) cudaFreeAsync(freq, s);
    if (pos) cudaFreeAsync(pos, s);
    tw32 = nullptr;
    tw64 = nullptr;
    freq = pos = nullptr;
  }
};

template <typename T> void* dalloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) return nullptr;
  dmalloc(&p, bytes);
  return p;
}

}  // namespace

// ------------------------------------------------------------ Engine<T> ----
// Everything that depends on the working precision T.
template <typename T> struct Engine {
  typedef typename C2<T>::t T2;
  bool on = false;
  T2* dc = nullptr;    // D octant
  T2* ccs = nullptr;   // [max_rhs][nmat][3] scaled sqrt(cc)
  T2* xhat = nullptr;  // [max_rhs][Gx][3][nlines]
  T2* zbuf = nullptr;  // split path [max_rhs][Gx][3][Gz][by]
  T2* vec[10] = {};    // Krylov vectors [max_rhs][3 nvs]
  T2* io = nullptr;    // host-API staging [max_rhs][3 nvs]
  T2* xo = nullptr;    // MIXED, FP64 engine: refined solution x and b = sqrt(cc) Einc
  T2* bo = nullptr;
  bool fused = false;
  int yz_groups = 1;          // fused kernel: thread groups per CTA (k.yz, k.yz2, k.yz4)
  bool yz_pair = false;       // fused path through k_yz_pair: a plane per cluster of two CTAs
  size_t pair_fixed = 0;      // k_yz_pair shared memory without the row buffers
  bool slot_path = false;     // k_yz_slot: cluster per plane through L2 slots
  T2* slots = nullptr;        // [ncl][Gz][wp]
  uint32_t* order = nullptr;  // kx positions, mirrored frequencies adjacent
  SlotGeom sg{};
  int ncl = 0, cl = 0;
  int ncl_by_cl[17] = {};     // resident clusters per cluster size (0: not schedulable)
  size_t yz_fixed = 0, yz_row = 0;  // fused kernel shared memory: fixed part, per row
  YzGeom yz{};
  size_t smem_x = 0, smem_yz = 0, smem_rows = 0, smem_cols = 0, smem_slot = 0;
  int tl = 1;                 // grid lines per k_xfwd / k_xinv tile
  ColGeom cz_fwd{}, cz_inv{};
  MvKernels<T> k;
  void release(cudaStream_t s) {
    for (void* p : {(void*)dc, (void*)ccs, (void*)xhat, (void*)zbuf, (void*)io, (void*)slots, (void*)order,
                    (void*)xo, (void*)bo})
      if (p) cudaFreeAsync(p, s);
    for (auto& v : vec)
      if (v) cudaFreeAsync(v, s);
    dc = ccs = xhat = zbuf = io = slots = xo = bo = nullptr;
    order = nullptr;
    for (auto& v : vec) v = nullptr;
  }
};

struct dda_ctx {
  std::atomic<int> cancel{0};  // dda_cancel: the running (or next) solve stops at its next round
  // MIXED: the FP64 engine's plane kernel shapes are tuned when a solve first
  // runs the FP64 convolution (many served targets never do)
  bool e64_tuned = true;
  int device = 0;
  int precision = DDA_PREC_FP64;
  int max_rhs = 1;
  uint32_t flags = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  MvGeom g{};
  double kd = 0, grid_unit = 0;
  uint32_t* line_off = nullptr;
  uint32_t* dip = nullptr;
  uint32_t* perm = nullptr;
  uint8_t* mat_ext = nullptr;
  FftPlan px, py, pz;  // runtime-engine plans (D-matrix setup, generic matvec)
  FftPlan mx, my, mz;  // matvec plans: tuned compile-time plans when `planned`
  bool planned = false;
  Engine<float> e32;
  Engine<double> e64;
  std::vector<std::complex<double>> cc_host;  // [max_rhs][nmat][3], reference units
  std::vector<char> cc_set;
  KrylovState* st = nullptr;  // device [max_rhs]
  KrylovState* st_host = nullptr;  // host mirror (pageable: freeing pinned memory may wait for the device)
  KrylovState* st_outer = nullptr;  // device: FP64 refinement loop (MIXED)
  KrylovState* sto_host = nullptr;  // host mirror
  RedSums* parts = nullptr;
  unsigned* tickets = nullptr;
  int nparts_vec = 0, nparts_mv = 0;
  double* hist = nullptr;
  long long hist_cap = 0;
  long long launches = 0;  // kernels this context has launched
  // instantiated graphs of one solver round, per (solver, nrhs, precision):
  // the round's kernel arguments are the context's fixed buffers
  struct RoundGraph {
    int solver, nrhs, tsize;
    cudaGraphExec_t g;
    long long launches;
  };
  std::vector<RoundGraph> round_graphs;
  size_t dev_bytes = 0;    // device memory held after dda_create

  // Frees on the context stream once its work is done; other contexts'
  // work on the device is not waited for.
  void release() {
    if (device >= 0) cudaSetDevice(device);
    for (auto& rg : round_graphs) cudaGraphExecDestroy(rg.g);
    round_graphs.clear();
    cudaStream_t s = stream;
    if (s) cudaStreamSynchronize(s);
    e32.release(s);
    e64.release(s);
    px.release(s);
    py.release(s);
    pz.release(s);
    mx.release(s);
    my.release(s);
    mz.release(s);
    for (void* p : {(void*)line_off, (void*)dip, (void*)perm, (void*)mat_ext, (void*)st,
                    (void*)parts, (void*)tickets, (void*)hist, (void*)st_outer})
      if (p) cudaFreeAsync(p, s);
    delete[] st_host;
    delete[] sto_host;
    st_outer = nullptr;
    sto_host = nullptr;
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    line_off = dip = perm = nullptr;
    mat_ext = nullptr;
    st = nullptr;
    st_host = nullptr;
    parts = nullptr;
    tickets = nullptr;
    hist = nullptr;
    stream = nullptr;
  }
};

namespace {

int ntiles(const dda_ctx* c, int tl) { return (c->g.nlines + tl - 1) / tl; }

// CTAs of the vector steps per right-hand side: every SM filled with as many
// as it holds of the heaviest step (QMR-CS update: six vector streams), at
// least 512 elements each.  A fixed function of the problem and the device,
// as the partial sums of the dot products follow it.
int vec_parts(dda_ctx* c) {
  int nsm = 148;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
  int occ = kVecPartsMax;
  auto limit = [&](auto fn) {
    int n = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kNtV, 0));
    occ = std::min(occ, std::max(1, n));
  };
  if (c->e32.on && c->precision == DDA_PREC_FP32) limit(k_vec<float, kNtV, V_QMR_UPD>);
  if (c->e64.on) limit(k_vec<double, kNtV, V_QMR_UPD>);
  const long long len = 3LL * c->g.nvs;
  const long long parts = std::min<long long>((long long)occ * nsm, (len + 511) / 512);
  return (int)std::max(1LL, std::min<long long>(parts, kVecPartsMax));
}

// Largest x tile (grid lines) whose shared memory stays within 72 KB, so
// that three CTAs of k_xfwd / k_xinv share an SM.
inline int x_tile_max(long long cbytes, long long Gx) {
  return (int)std::max(1LL, std::min((long long)kXTileMax, 73728 / (cbytes * (Gx + 1))));
}

template <typename T> Engine<T>& eng(dda_ctx* c);
template <> Engine<float>& eng<float>(dda_ctx* c) { return c->e32; }
template <> Engine<double>& eng<double>(dda_ctx* c) { return c->e64; }

// Clusters of `cl` CTAs of k_yz_slot with `smem` bytes each that fit the
// device at once (0 when the shape cannot be scheduled).
template <typename T> int slot_clusters(Engine<T>& e, int cl, size_t smem) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(cl);
  cfg.blockDim = dim3(kNtYz);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (const void*)e.k.slot, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// k_yz_slot set-up: row batch, cluster size, resident clusters, one slot per
// cluster, and the kx order that puts the planes kx and -kx (one D-hat
// octant plane) next to each other.  Leaves e.slot_path false when the
// cluster shape cannot be scheduled (the split path then runs).
template <typename T> void setup_slot(dda_ctx* c, Engine<T>& e) {
  typedef typename C2<T>::t T2;
  const MvGeom& g = c->g;
  SlotGeom sg;
  sg.wp = (3 * g.by + 31) / 32 * 32;
  sg.py = g.Gy + 1;
  const int cl = 8;  // default shape; autotune may pick 4 or 16
  int nrw = std::min(16, (g.Gz + cl - 1) / cl);
  while (nrw > 1 && slot_smem_bytes<T>(g, nrw) > kSmemMax) nrw--;
  sg.nrw = nrw;
  const size_t smem = slot_smem_bytes<T>(g, nrw);
  if (smem > kSmemMax) return;
  CK(allow_smem((const void*)e.k.slot));
  CK(cudaFuncSetAttribute((const void*)e.k.slot, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  int ncl_max = 0;
  for (int cand : {4, 8, 16}) {
    e.ncl_by_cl[cand] = std::min(slot_clusters<T>(e, cand, slot_smem_bytes<T>(g, 1)), g.Gx * c->max_rhs);
    ncl_max = std::max(ncl_max, e.ncl_by_cl[cand]);
  }
  int ncl = std::min(slot_clusters<T>(e, cl, smem), g.Gx * c->max_rhs);
  if (ncl < 1) return;
  std::vector<uint32_t> order;
  for (int f = 0; f <= g.Gx / 2; f++) {
    order.push_back((uint32_t)c->mx.pos_h[f]);
    if (f != 0 && f != g.Gx / 2) order.push_back((uint32_t)c->mx.pos_h[g.Gx - f]);
  }
  e.order = (uint32_t*)dalloc<float>(order.size() * sizeof(uint32_t));
  CK(cudaMemcpyAsync(e.order, order.data(), order.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
  e.slots = (T2*)dalloc<T>((size_t)ncl_max * g.Gz * sg.wp * sizeof(T2));
  e.sg = sg;
  e.cl = cl;
  e.ncl = ncl;
  e.smem_slot = smem;
  e.slot_path = true;
}

// Group count forced by the context flags (1: none).
inline int forced_groups(uint32_t flags) {
  if (flags & DDA_FLAG_YZ_GROUPS4) return 4;
  if (flags & DDA_FLAG_YZ_GROUPS2) return 2;
  return 1;
}

// The fused plane kernel run as `groups` thread groups (nullptr: none).
template <typename T> typename MvKernels<T>::YzFn fused_yz(const Engine<T>& e, int groups) {
  switch (groups) {
    case 1: return e.k.yz;
    case 2: return e.k.yz2;
    case 4: return e.k.yz4;
    default: return nullptr;
  }
}

// Every x-pass kernel of an engine (plain, with a solver step in the load,
// over FP64 vectors).
template <typename T> std::vector<const void*> x_pass_kernels(const Engine<T>& e) {
  std::vector<const void*> v;
  for (const void* f : {(const void*)e.k.xfwd, (const void*)e.k.xfwd_pre, (const void*)e.k.xinv,
                        (const void*)e.k.xfwd_m, (const void*)e.k.xfwd_m_pre, (const void*)e.k.xinv_m})
    if (f) v.push_back(f);
  return v;
}

// Lines per k_xfwd / k_xinv tile.  The two x passes launch
// ntiles x 3 x nrhs CTAs of a few microseconds each, so the count of waves
// over the SMs decides their time: among tiles from half the 72 KB maximum
// up to it, the one with the least (waves x (lines + 2)) wins, the 2 lines
// standing for a CTA's fixed cost (twiddles, material table).  Depends on the
// grid, the box, max_rhs and the device only, never on timing, so that a
// problem's arithmetic (the partial sums of the fused dot products follow
// the tiles) is the same in every context that solves it.
template <typename T> void pick_x_tile(dda_ctx* c, Engine<T>& e) {
  const MvGeom& g = c->g;
  const size_t s = sizeof(typename C2<T>::t);
  int nsm = 148;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
  const std::vector<const void*> xk = x_pass_kernels(e);
  for (const void* f : xk) CK(allow_smem(f));
  const int tmax = x_tile_max((long long)s, g.Gx);
  long long best_cost = -1;
  for (int tl = std::max(1, tmax / 2); tl <= tmax; tl++) {
    const size_t smem = ((size_t)g.Gx + g.nmat + (size_t)tl * g.pitchx) * s;
    int occ = 1 << 30;  // the least over every x-pass variant
    for (const void* f : xk) {
      int o = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, f, kNtX, smem));
      occ = std::min(occ, o);
    }
    const long long slots = (long long)std::max(1, occ) * nsm;
    const long long ctas = (long long)ntiles(c, tl) * 3 * c->max_rhs;
    const long long cost = (ctas + slots - 1) / slots * (tl + 2);
    if (best_cost < 0 || cost <= best_cost) {
      best_cost = cost;
      e.tl = tl;
    }
  }
  // twiddles, material table, tile of tl lines x (Gx+1)
  e.smem_x = ((size_t)g.Gx + g.nmat + (size_t)e.tl * g.pitchx) * s;
}

// Chooses tile shapes and allocates the matvec buffers of one precision.
template <typename T> void setup_engine(dda_ctx* c) {
  typedef typename C2<T>::t T2;
  Engine<T>& e = eng<T>(c);
  const MvGeom& g = c->g;
  const size_t s = sizeof(T2);
  e.on = true;
  constexpr int NW = kNtYz / 32;
  // fused plane kernel: twiddles, slab Gz x q, row buffers 3 x (Gy+1)
  YzGeom y;
  y.q = 3 * g.by + ((3 * g.by) % 2 == 0 ? 1 : 0);
  y.py = g.Gy + 1;
  const size_t fixed = ((size_t)g.Gz + g.Gy + (size_t)g.Gz * y.q) * s;
  const size_t row = (size_t)3 * y.py * s;
  e.k = select_kernels<T>(c->planned, g.Gx, g.Gy, g.Gz, g.by, g.bz);
  // row buffers: one per warp in the runtime-planned kernel, batches of up
  // to 32 rows in the planned one
  int nrw = c->planned ? 32 : NW;
  while (nrw > 1 && fixed + nrw * row > kSmemMax) nrw--;
  y.nrw = nrw;
  e.yz = y;
  e.smem_yz = fixed + nrw * row;
  e.yz_fixed = fixed;
  e.yz_row = row;
  e.fused = e.k.yz && e.smem_yz <= kSmemMax && !(c->flags & (DDA_FLAG_SPLIT_YZ | DDA_FLAG_SLOT_YZ));
  // the two-CTA plane kernel: an autotuner candidate where one CTA holds a
  // plane, the path where only half a plane fits (FP64 planes of the fused
  // lengths: 1.2-1.8x faster than the cluster kernel's L2 slots), and forced
  // by DDA_FLAG_YZ_PAIR
  e.pair_fixed = ((size_t)g.Gz + g.Gy + (size_t)(g.Gz / 2) * y.q) * s;
  const bool pair_fits = e.k.pair[0] && e.pair_fixed + 4 * row <= kSmemMax &&
                         !(c->flags & (DDA_FLAG_SPLIT_YZ | DDA_FLAG_SLOT_YZ));
  if (pair_fits && ((c->flags & DDA_FLAG_YZ_PAIR) || !e.fused)) {
    int np = 32;
    while (np > 1 && e.pair_fixed + np * row > kSmemMax) np--;
    e.fused = true;
    e.yz_pair = true;
    e.yz.nrw = np;
    e.smem_yz = e.pair_fixed + np * row;
  }
  const int forced = forced_groups(c->flags);
  if (e.yz_pair && forced > 1 && e.yz.nrw >= forced) {
    e.yz_groups = forced;
    e.yz.nrw -= e.yz.nrw % forced;
    e.smem_yz = e.pair_fixed + e.yz.nrw * row;
  }
  if (e.fused && !e.yz_pair && forced > 1 && fused_yz<T>(e, forced) && nrw >= forced) {
    e.yz_groups = forced;
    e.yz.nrw = nrw - nrw % forced;  // a multiple of the groups: an equal share each
    e.smem_yz = fixed + e.yz.nrw * row;
  }
  if (!e.fused && e.k.slot && !(c->flags & DDA_FLAG_SPLIT_YZ)) setup_slot<T>(c, e);
  if (!e.fused && !e.slot_path) {
    // split path: zbuf, k_yrows over NW rows per CTA, column FFTs along z
    e.yz.nrw = NW;
    e.smem_rows = ((size_t)g.Gy + (size_t)NW * 3 * y.py) * s;
    int ti = std::min(32, g.by);
    while (ti > 1 && ((size_t)g.Gz + (size_t)g.Gz * (ti + 1)) * s > kSmemMax) ti--;
    e.smem_cols = ((size_t)g.Gz + (size_t)g.Gz * (ti + 1)) * s;
    ColGeom f;
    f.in_bs = g.nlines;            // xhat plane of one component
    f.in_as = g.by;
    f.out_bs = (long long)g.Gz * g.by;
    f.out_as = g.by;
    f.inner = g.by;
    f.ti = ti;
    f.pitch = ti + 1;
    f.n_in = g.bz;
    f.n_out = g.Gz;
    f.batches_per_rhs = g.Gx * 3;
    e.cz_fwd = f;
    ColGeom iv = f;
    iv.in_bs = f.out_bs;
    iv.in_as = g.by;
    iv.out_bs = g.nlines;
    iv.out_as = g.by;
    iv.n_in = g.Gz;
    iv.n_out = g.bz;
    e.cz_inv = iv;
    if (e.smem_rows > kSmemMax || e.smem_cols > kSmemMax)
      throw DdaError(DDA_ERR_UNSUPPORTED, "FFT grid too large for the shared-memory tiles");
    e.zbuf = (T2*)dalloc<T>((size_t)c->max_rhs * g.Gx * 3 * g.Gz * g.by * s);
  }
  pick_x_tile<T>(c, e);
  if (e.smem_x > kSmemMax) throw DdaError(DDA_ERR_UNSUPPORTED, "grid x extent too large");
  auto attr = [](const void* f, size_t bytes) {
    if (bytes > kSmemMax) throw DdaError(DDA_ERR_UNSUPPORTED, "shared-memory tile above the SM limit");
    CK(allow_smem(f));
  };
  for (const void* f : x_pass_kernels(e)) attr(f, e.smem_x);
  if (e.fused) {
    for (int gr : {1, 2, 4})
      if (fused_yz<T>(e, gr)) attr((const void*)fused_yz<T>(e, gr), e.smem_yz);
    for (auto f : e.k.pair)
      if (f) attr((const void*)f, e.smem_yz);
  }
  else if (!e.slot_path) {
    attr((const void*)e.k.yrows, e.smem_rows);
    attr((const void*)e.k.cols, e.smem_cols);
  }
  const int hx = g.Gx / 2 + 1, hy = g.Gy / 2 + 1, hz = g.Gz / 2 + 1;
  e.dc = (T2*)dalloc<T>((size_t)hx * hy * hz * 6 * s);
  e.ccs = (T2*)dalloc<T>((size_t)c->max_rhs * g.nmat * 3 * s);
  CK(cudaMemsetAsync(e.ccs, 0, (size_t)c->max_rhs * g.nmat * 3 * s, c->stream));
  e.xhat = (T2*)dalloc<T>((size_t)c->max_rhs * g.Gx * 3 * g.nlines * s);
  const size_t vbytes = (size_t)c->max_rhs * 3 * g.nvs * s;
  // a MIXED context runs its Krylov vectors in FP64 and only the matvec's
  // convolution in FP32: the FP32 engine needs one input buffer and io
  const bool conv_engine = c->precision == DDA_PREC_MIXED && sizeof(T) == 4;
  for (int i = 0; i < 10; i++) {
    if (conv_engine && i > 0) break;
    e.vec[i] = (T2*)dalloc<T>(vbytes);
    CK(cudaMemsetAsync(e.vec[i], 0, vbytes, c->stream));
  }
  e.io = (T2*)dalloc<T>(vbytes);
  if (c->precision == DDA_PREC_MIXED && sizeof(T) == 8) {
    e.xo = (T2*)dalloc<T>(vbytes);
    e.bo = (T2*)dalloc<T>(vbytes);
  }
}

// Uploads the scaled couple constants of every rhs to the engine.
template <typename T> void upload_cc(dda_ctx* c) {
  typedef typename C2<T>::t T2;
  Engine<T>& e = eng<T>(c);
  if (!e.on) return;
  const double sc = std::pow(c->grid_unit, -1.5);
  std::vector<T2> h(c->cc_host.size());
  for (size_t i = 0; i < h.size(); i++) {
    h[i].x = (T)(c->cc_host[i].real() * sc);
    h[i].y = (T)(c->cc_host[i].imag() * sc);
  }
  CK(cudaMemcpyAsync(e.ccs, h.data(), h.size() * sizeof(T2), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

RedTarget red_target(dda_ctx* c, int nparts) {
  RedTarget t;
  t.parts = c->parts;
  t.tickets = c->tickets;
  t.nparts = nparts;
  return t;
}

// The y/z passes: the fused plane kernel, the cluster kernel, or the split
// path (column FFTs along z around the row kernel).
template <typename T>
void launch_yz(dda_ctx* c, int nrhs, cudaStream_t s, KrylovState* st, int skipmv) {
  Engine<T>& e = eng<T>(c);
  const MvGeom& g = c->g;
  const FftPlanDev py = c->my.dev<T>(), pz = c->mz.dev<T>();
  if (e.fused && e.yz_pair) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(2 * g.Gx, nrhs);
    cfg.blockDim = dim3(kNtYz);
    cfg.dynamicSmemBytes = e.smem_yz;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const auto f = e.k.pair[e.yz_groups == 4 ? 2 : e.yz_groups == 2 ? 1 : 0];
    CK(cudaLaunchKernelEx(&cfg, f, e.xhat, (const typename C2<T>::t*)e.dc, g, e.yz, pz, py, (const KrylovState*)st,
                          skipmv));
  } else if (e.fused) {
    fused_yz<T>(e, e.yz_groups)<<<dim3(g.Gx, nrhs), kNtYz, e.smem_yz, s>>>(e.xhat, e.dc, g, e.yz, pz, py, st,
                                                                           skipmv);
  } else if (e.slot_path) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = e.cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(std::min(e.ncl, g.Gx * nrhs) * e.cl);
    cfg.blockDim = dim3(kNtYz);
    cfg.dynamicSmemBytes = e.smem_slot;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, e.k.slot, e.xhat, (const typename C2<T>::t*)e.dc, g, e.sg,
                          (const uint32_t*)e.order, nrhs, e.slots, pz, py, (const KrylovState*)st, skipmv));
  } else {
    const int nbatch = nrhs * g.Gx * 3;
    dim3 gc((g.by + e.cz_fwd.ti - 1) / e.cz_fwd.ti, nbatch);
    e.k.cols<<<gc, kNtC, e.smem_cols, s>>>(e.xhat, e.zbuf, e.cz_fwd, pz, 0, st, skipmv);
    dim3 gr((g.Gz + e.yz.nrw - 1) / e.yz.nrw, g.Gx, nrhs);
    e.k.yrows<<<gr, kNtYz, e.smem_rows, s>>>(e.zbuf, e.dc, g, e.yz, py, st, skipmv);
    e.k.cols<<<gc, kNtC, e.smem_cols, s>>>(e.zbuf, e.xhat, e.cz_inv, pz, 1, st, skipmv);
  }
}

// ------------------------------------------------------------ autotune ----
// Shape parameters of the y/z passes that do not change the arithmetic (each
// plane and row is transformed the same way whatever the batching), chosen
// by timing: the fused kernel's rows per batch, the cluster kernel's cluster
// size and rows per batch.  Timed on the context's own buffers (x spectrum
// zeroed, one right-hand side) and kept per shape for the process.
struct TuneChoice {
  int nrw = 0, cl = 0, groups = 1, pair = 0;
  int ncl = 0;  // cluster kernel: clusters in flight (0: as many as can be resident)
};
std::mutex g_tune_mu;
std::map<std::array<int, 8>, TuneChoice> g_tune_cache;

template <typename T> float time_yz(dda_ctx* c, int nrhs, int reps) {
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  launch_yz<T>(c, nrhs, c->stream, nullptr, 0);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < reps; r++) {
    CK(cudaEventRecord(a, c->stream));
    launch_yz<T>(c, nrhs, c->stream, nullptr, 0);
    CK(cudaEventRecord(b, c->stream));
    CK(cudaEventSynchronize(b));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    best = std::min(best, ms);
  }
  CK(cudaGetLastError());
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

template <typename T> void apply_choice(dda_ctx* c, Engine<T>& e, const TuneChoice& t) {
  const MvGeom& g = c->g;
  if (e.fused) {
    e.yz.nrw = t.nrw;
    e.yz_groups = t.groups;
    e.yz_pair = t.pair != 0;
    e.smem_yz = (e.yz_pair ? e.pair_fixed : e.yz_fixed) + (size_t)t.nrw * e.yz_row;
  } else if (e.slot_path) {
    e.cl = t.cl;
    e.ncl = t.ncl > 0 ? std::min(t.ncl, e.ncl_by_cl[t.cl]) : e.ncl_by_cl[t.cl];
    e.sg.nrw = t.nrw;
    e.smem_slot = slot_smem_bytes<T>(g, t.nrw);
  }
}

template <typename T> void autotune(dda_ctx* c) {
  Engine<T>& e = eng<T>(c);
  const MvGeom& g = c->g;
  if (!e.on || !(e.fused || e.slot_path)) return;
  NvtxRange range(sizeof(T) == 4 ? "dda autotune fp32" : "dda autotune fp64");
  if ((long long)g.Gx * g.Gy * g.Gz < (1LL << 20)) return;  // small grids keep the defaults
  // the box changes the best batching little next to the grid, so shapes
  // share a choice per grid (served targets mostly land on tuned grids)
  // (the flags that restrict the candidates are part of the shape)
  const std::array<int, 8> key = {g.Gx, g.Gy, g.Gz, (int)sizeof(T), c->planned ? 1 : 0, e.fused ? 0 : 1,
                                   std::min(c->max_rhs, 4),
                                   forced_groups(c->flags) + (c->flags & DDA_FLAG_YZ_PAIR ? 100 : 0)};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      apply_choice<T>(c, e, it->second);
      return;
    }
  }
  std::vector<TuneChoice> cands;
  if (e.fused) {
    const int max_rows = e.k.planned ? 48 : kNtYz / 32;
    for (int n : {4, 6, 8, 10, 12, 14, 16, 20, 24, 25, 28, 32, 34, 36, 40, 43, 48})
      if (n <= max_rows && e.yz_fixed + (size_t)n * e.yz_row <= kSmemMax) {
        if (c->flags & DDA_FLAG_YZ_PAIR) continue;
        const int forced = forced_groups(c->flags);
        // gr groups of n / gr rows each (a forced group count keeps only it)
        for (int gr : {1, 2, 4})
          if (fused_yz<T>(e, gr) && n % gr == 0 && (forced == 1 || gr == forced)) cands.push_back({n, 0, gr, 0});
      }
    // the two-CTA plane kernel: half the slab per CTA, more rows
    if (e.k.pair[0] && forced_groups(c->flags) == 1)
      for (int n : {8, 12, 16, 20, 24, 28, 32, 36, 40, 48})
        if (n <= 48 && n <= g.Gz / 2 && e.pair_fixed + (size_t)n * e.yz_row <= kSmemMax)
          for (int gr : {1, 2, 4})
            if (n % gr == 0) cands.push_back({n, 0, gr, 1});
  } else {
    int l2 = 0;
    CK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, c->device));
    const size_t slot_bytes = (size_t)g.Gz * e.sg.wp * sizeof(typename C2<T>::t);
    for (int cl : {4, 8, 16})
      for (int n : {4, 8, 16})
        if (e.ncl_by_cl[cl] > 0 && n <= (g.Gz + cl - 1) / cl && slot_smem_bytes<T>(g, n) <= kSmemMax &&
            slot_clusters<T>(e, cl, slot_smem_bytes<T>(g, n)) >= e.ncl_by_cl[cl]) {
          cands.push_back({n, cl});
          // fewer clusters in flight: their plane buffers then stay in L2
          // next to the streamed planes, at the price of less latency hiding
          // -- worth timing only where the buffers of all clusters fill more
          // than half the L2 (each candidate costs context set-up time)
          if ((size_t)e.ncl_by_cl[cl] * slot_bytes * 2 <= (size_t)l2) continue;
          for (int div : {2, 3})
            if (e.ncl_by_cl[cl] / div >= 4) {
              TuneChoice t{n, cl};
              t.ncl = e.ncl_by_cl[cl] * (div - 1) / div;
              cands.push_back(t);
            }
        }
  }
  if (cands.size() < 2) return;
  // timed on up to four right-hand sides: with one, a launch is about a wave
  // of CTAs and the tail decides; with several, the steady rate does, as in
  // the solves of batched contexts
  const int nt = std::min(c->max_rhs, 4);
  CK(cudaMemsetAsync(e.xhat, 0, (size_t)nt * g.Gx * 3 * g.nlines * sizeof(typename C2<T>::t), c->stream));
  TuneChoice best = cands[0];
  float best_ms = 1e30f;
  for (const TuneChoice& t : cands) {
    apply_choice<T>(c, e, t);
    const float ms = time_yz<T>(c, nt, 2);
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  apply_choice<T>(c, e, best);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = best;
}

// The matvec: k_xfwd -> (k_yz | k_yz_slot | cols/yrows/cols) -> k_xinv, over
// vectors of element type A2: the engine's own (T = float or double), or
// FP64 vectors around the FP32 convolution (T = float, A2 = double2: the
// argument is rounded to FP32 as k_xfwd reads it, the identity term added in
// FP64 by k_xinv).  pre: a solver step that produces the argument, run in
// k_xfwd's load (arg is then pre.out).
template <typename T, typename A2 = typename C2<T>::t>
void matvec(dda_ctx* c, const A2* arg, A2* res, int conj, int nrhs, cudaStream_t s, KrylovState* st,
            KrylovStep step, int skipmv = 0, XPre pre = XPre{}) {
  Engine<T>& e = eng<T>(c);
  MvGeom g = c->g;
  g.tl = e.tl;
  const FftPlanDev px = c->mx.dev<T>();
  dim3 gx(ntiles(c, e.tl), 3, nrhs);
  const RedTarget red = red_target(c, 3 * ntiles(c, e.tl));
  typename MvKernels<T>::template XfwdF<A2> xf;
  typename MvKernels<T>::template XinvF<A2> xi;
  if constexpr (std::is_same<A2, typename C2<T>::t>::value) {
    xf = pre.op != XP_NONE ? e.k.xfwd_pre : e.k.xfwd;
    xi = e.k.xinv;
  } else {
    xf = pre.op != XP_NONE ? e.k.xfwd_m_pre : e.k.xfwd_m;
    xi = e.k.xinv_m;
  }
  if (pre.op != XP_NONE) {
    pre.out = const_cast<A2*>(arg);
    pre.step.red = red;
  }
  xf<<<gx, kNtX, e.smem_x, s>>>(arg, e.xhat, c->line_off, c->dip, c->perm, e.ccs, conj, g, px, st, skipmv, pre);
  launch_yz<T>(c, nrhs, s, st, skipmv);
  step.red = red;
  xi<<<gx, kNtX, e.smem_x, s>>>(arg, res, e.xhat, c->line_off, c->dip, c->perm, e.ccs, conj, g, px, st, step, skipmv);
  CK(cudaGetLastError());
  c->launches += (e.fused || e.slot_path) ? 3 : 5;
}

// D-matrix generation (FP64) into the enabled engines' octants.
void build_dmatrix(dda_ctx* c) {
  NvtxRange range("dda D matrix");
  const MvGeom& g = c->g;
  const long long N = (long long)g.Gx * g.Gy * g.Gz;
  double2* full = nullptr;
  CK(cudaMallocAsync(&full, N * sizeof(double2), c->stream));
  const FftPlanDev px = c->px.dev<double>(), py = c->py.dev<double>(), pz = c->pz.dev<double>();
  CK(allow_smem((const void*)k_fft_rows<double, kNtC>));
  CK(allow_smem((const void*)k_fft_cols<double, kNtC>));
  static const int MU[6] = {0, 0, 0, 1, 1, 2}, NU[6] = {0, 1, 2, 1, 2, 2};
  int tlr = 32;
  while (tlr > 1 && ((size_t)g.Gx + (size_t)tlr * (g.Gx + 1)) * sizeof(double2) > kSmemMax) tlr--;
  const size_t smr = ((size_t)g.Gx + (size_t)tlr * (g.Gx + 1)) * sizeof(double2);
  auto cols = [&](const FftPlanDev& pl, long long inner, long long batch, long long bs, long long as) {
    const int n = pl.n;
    int ti = (int)std::min<long long>(32, inner);
    while (ti > 1 && ((size_t)n + (size_t)n * (ti + 1)) * sizeof(double2) > kSmemMax) ti--;
    ColGeom cg;
    cg.in_bs = bs; cg.in_as = as; cg.out_bs = bs; cg.out_as = as;
    cg.inner = (int)inner; cg.ti = ti; cg.pitch = ti + 1;
    cg.n_in = n; cg.n_out = n;
    cg.batches_per_rhs = 1;
    const size_t sm = ((size_t)n + (size_t)n * (ti + 1)) * sizeof(double2);
    if (sm > kSmemMax) throw DdaError(DDA_ERR_UNSUPPORTED, "grid too large for D-matrix FFT tiles");
    k_fft_cols<double, kNtC><<<dim3((unsigned)((inner + ti - 1) / ti), (unsigned)batch), kNtC, sm, c->stream>>>(
        full, full, cg, pl, 0, nullptr, 0);
  };
  for (int comp = 0; comp < 6; comp++) {
    k_dfill<<<1184, 256, 0, c->stream>>>(full, g.Gx, g.Gy, g.Gz, g.bx, g.by, g.bz, c->kd, MU[comp], NU[comp]);
    k_fft_rows<double, kNtC><<<(unsigned)(((long long)g.Gy * g.Gz + tlr - 1) / tlr), kNtC, smr, c->stream>>>(
        full, (long long)g.Gy * g.Gz, g.Gx, tlr, g.Gx + 1, px, 0);
    cols(py, g.Gx, g.Gz, (long long)g.Gy * g.Gx, g.Gx);
    cols(pz, (long long)g.Gy * g.Gx, 1, N, (long long)g.Gy * g.Gx);
    k_dcompress<<<592, 256, 0, c->stream>>>(full, c->e64.on ? c->e64.dc : nullptr,
                                            c->e32.on ? c->e32.dc : nullptr, g.Gx, g.Gy, g.Gz, comp,
                                            c->px.pos, c->py.pos, c->pz.pos);
    CK(cudaGetLastError());
  }
  CK(cudaFreeAsync(full, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

// Host-supplied D (reference layout, reference units) -> octants.
void upload_dmatrix(dda_ctx* c, const double* D) {
  const MvGeom& g = c->g;
  const int hx = g.Gx / 2 + 1, hy = g.Gy / 2 + 1, hz = g.Gz / 2 + 1;
  const double sc = c->grid_unit * c->grid_unit * c->grid_unit;
  std::vector<double2> h64((size_t)hx * hy * hz * 6);
  for (int ax = 0; ax < hx; ax++)
    for (int az = 0; az < hz; az++)
      for (int ay = 0; ay < hy; ay++)
        for (int comp = 0; comp < 6; comp++) {
          const size_t src = comp + 6 * (ay + (size_t)g.Gy * (az + (size_t)g.Gz * ax));
          const size_t dst = (((size_t)ax * hz + az) * hy + ay) * 6 + comp;
          h64[dst] = make_double2(D[2 * src] * sc, D[2 * src + 1] * sc);
        }
  double2* tmp = nullptr;
  CK(cudaMallocAsync(&tmp, h64.size() * sizeof(double2), c->stream));
  CK(cudaMemcpyAsync(tmp, h64.data(), h64.size() * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  if (c->e64.on)
    CK(cudaMemcpyAsync(c->e64.dc, tmp, h64.size() * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
  if (c->e32.on) {
    k_d64_to_d32<<<592, 256, 0, c->stream>>>(tmp, c->e32.dc, (long long)h64.size());
    CK(cudaGetLastError());
  }
  CK(cudaFreeAsync(tmp, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

int fail(dda_ctx* c, const DdaError& e) {
  if (c) c->err = e.what();
  else g_create_error = e.what();
  return e.code;
}

template <typename F> int guard(dda_ctx* c, F f) {
  try {
    if (c) CK(cudaSetDevice(c->device));
    return f();
  } catch (const DdaError& e) {
    return fail(c, e);
  } catch (const std::exception& e) {
    return fail(c, DdaError(DDA_ERR_ARG, e.what()));
  }
}

}  // namespace

// ============================================================ solver ======
namespace {

template <typename T> struct Solve {
  typedef typename C2<T>::t T2;
  dda_ctx* c;
  Engine<T>& e;
  int nrhs;
  cudaStream_t s;
  KrylovState* st;
  Solve(dda_ctx* c_, int nrhs_, KrylovState* st_ = nullptr)
      : c(c_), e(eng<T>(c_)), nrhs(nrhs_), s(c_->stream), st(st_ ? st_ : c_->st) {}

  KrylovStep step(int op, int mode = EP_NORM, const void* w = nullptr, int nparts = 0) {
    KrylovStep k;
    k.op = op;
    k.mode = mode;
    k.w = w;
    k.red = red_target(c, nparts ? nparts : c->nparts_vec);
    return k;
  }

  void vec(int op, int first, std::initializer_list<T2*> v, KrylovStep k) {
    VecArgs a;
    memset(&a, 0, sizeof(a));
    int i = 0;
    for (T2* p : v) a.v[i++] = p;
    a.op = op;
    a.first = first;
    a.nv = c->g.nv;
    a.nvs = c->g.nvs;
    a.nmat = c->g.nmat;
    a.nparts = c->nparts_vec;
    a.mat = c->mat_ext;
    a.ccs = e.ccs;
    a.pscale = c->grid_unit * c->grid_unit * c->grid_unit;
    a.step = k;
    vec_kernel<T, kNtV>(a.op)<<<dim3(c->nparts_vec, nrhs), kNtV, 0, s>>>(a, st);
    CK(cudaGetLastError());
    c->launches++;
  }

  // FP64 Krylov vectors with the convolution of the matvec in FP32 (MIXED
  // inner solves): arg -> FP32, convolution sqrt(cc) IFFT(D FFT(sqrt(cc) .)),
  // then y = arg + conv and the step's sums in FP64.
  bool mv32 = false;

  void matvec_any(const T2* arg, T2* res, int conj, KrylovStep k, int skipmv = 0, XPre pre = XPre{}) {
    if constexpr (std::is_same<T, double>::value) {
      if (mv32) {
        matvec<float, double2>(c, arg, res, conj, nrhs, s, st, k, skipmv, pre);
        return;
      }
    }
    matvec<T>(c, arg, res, conj, nrhs, s, st, k, skipmv, pre);
  }

  void mv(const T2* arg, T2* res, int conj, KrylovStep k) { matvec_any(arg, res, conj, k); }

  // res = A out, with out = the solver step `op` of v1, v2 (and out) computed
  // in the matvec's first pass (XPreOp); pk: its sums, if any.
  void mv_pre(int op, int first, T2* out, const T2* v1, const T2* v2, T2* res, KrylovStep pk, KrylovStep k,
              int skipmv = 0) {
    XPre pre{};
    pre.op = op;
    pre.first = first;
    pre.v1 = v1;
    pre.v2 = v2;
    pre.step = pk;
    matvec_any(out, res, 0, k, skipmv, pre);
  }

  // CpuIterativeSolver::initGeneral (DDA/CpuIterativeSolver.cpp:45-91) with
  // the GPU setup kernels of DDA/GpuIterativeSolver.cpp:78-134.
  void init_general(T2* E, T2* B, T2* R, T2* X, T2* A, T2* S, bool start, bool b_given = false) {
    if (b_given) vec(V_NORM, 0, {B}, step(KOP_INIT_PVEC));
    else vec(V_SETUP_PVEC, 0, {B, E}, step(KOP_INIT_PVEC));
    if (start) {
      vec(V_START_X, 0, {X, S}, KrylovStep{KOP_NONE, 0, nullptr, {}});
      mv(X, A, 0, step(KOP_NONE));
      vec(V_R_INIT, 0, {R, A, B}, step(KOP_INIT_START));
    } else {
      mv(B, A, 0, step(KOP_NONE));
      vec(V_R_INIT, 0, {R, A, B}, step(KOP_INIT_R));
      vec(V_CHOOSE_X0, 0, {X, R, B}, step(KOP_NONE));
    }
  }

  // One iteration nr of the selected solver (buffers rotate on the host).
  struct Bufs {
    T2 *R, *X, *A, *t1, *t2, *t3, *t4;
  };
  void iteration(int solver, long long nr, Bufs& b) {
    switch (solver) {
      case DDA_SOLVER_QMR: {  // t1 = v, t2 = vt, t3 = p_old, t4 = p_new
        mv(b.t1, b.A, 0, step(KOP_QMR_ALPHA, EP_YA_BIL));
        vec(V_QMR_VT, nr == 0, {b.t2, b.t1, b.A}, step(KOP_QMR_GIVENS));
        vec(V_QMR_UPD, nr == 0 ? 1 : nr == 1 ? 2 : 0, {b.R, b.t3, b.t4, b.t1, b.t2, b.X}, step(KOP_QMR_END));
        if (nr > 0) std::swap(b.t3, b.t4);
        std::swap(b.t1, b.t2);
        break;
      }
      case DDA_SOLVER_BICGSTAB: {  // t1 = p, t2 = v, t3 = s, t4 = rt
        // p = r + beta (p - omega v) and s = r - alpha v run in the first
        // pass of the matvec they feed; the s step's |s|^2 decides the
        // half-step exit, which the rest of that matvec then skips
        mv_pre(XP_BIS_P, nr == 0, b.t1, b.t2, b.R, b.t2, step(KOP_NONE), step(KOP_BIS_ALPHA, EP_YW_HERM, b.t4));
        mv_pre(XP_BIS_S, 0, b.t3, b.t2, b.R, b.A, step(KOP_BIS_S), step(KOP_BIS_OMEGA, EP_AY_HERM_NORM), 1);
        vec(V_BIS_XR, 0, {b.X, b.t1, b.t3, b.A, b.R, b.t4}, step(KOP_BIS_END));
        break;
      }
      case DDA_SOLVER_BICG: {  // t1 = p
        mv_pre(XP_BICG_P, nr == 0, b.t1, b.R, nullptr, b.A, step(KOP_NONE), step(KOP_BICG_MU, EP_YA_BIL));
        vec(V_BICG_XR, 0, {b.X, b.t1, b.A, b.R}, step(KOP_BICG_END));
        break;
      }
      default: {  // CGNR, t1 = p
        if (nr == 0) {
          mv(b.R, b.t1, 1, step(KOP_CGNR_RO, EP_NORM));
          mv(b.t1, b.A, 0, step(KOP_CGNR_ALPHA, EP_NORM));
        } else {
          mv(b.R, b.A, 1, step(KOP_CGNR_RO, EP_NORM));
          mv_pre(XP_CGNR_P, 0, b.t1, b.A, nullptr, b.A, step(KOP_NONE), step(KOP_CGNR_ALPHA, EP_NORM));
        }
        vec(V_CGNR_XR, 0, {b.X, b.t1, b.A, b.R}, step(KOP_CGNR_END));
        break;
      }
    }
  }

  void solver_init(int solver, Bufs& b) {
    switch (solver) {
      case DDA_SOLVER_QMR:
        vec(V_BICG_RO, 0, {b.R}, step(KOP_QMR_INIT));
        vec(V_QMR_V0, 0, {b.t1, b.R}, step(KOP_NONE));
        break;
      case DDA_SOLVER_BICGSTAB:
        vec(V_BIS_INIT, 0, {b.t4, b.R}, step(KOP_BIS_RO));
        break;
      case DDA_SOLVER_BICG:
        vec(V_BICG_RO, 0, {b.R}, step(KOP_BICG_RO));
        break;
      default:
        break;
    }
  }
};

const long long kMaxResIncrease[4] = {50000, 30000, 50000, 10};

struct SolveOpts {
  bool start = false;              // S holds start polarisations
  bool b_given = false;            // B already holds b (no sqrt(cc) Einc product)
  const double* eps_rhs = nullptr; // per-rhs relative residual targets
  const char* skip = nullptr;      // rhs left untouched (marked done from the start)
  bool result = true;              // write P = sqrt(cc) x to the engine's io buffer
  long long max_res_increase = 0;  // > 0: stagnation limit instead of the solver's
  long long rate_window = 0;       // > 0: stop when |r| does not halve in this many iterations
  bool mv32 = false;               // FP64 solve with the matvec convolution in FP32
  // MIXED inner solves (mv32): every check_every iterations the FP64
  // residual of the current iterate, |B - A x|^2 with the full FP64 matvec,
  // is compared with the recurrence's |r|^2.  A right-hand side ends when
  // the FP64 residual is below check_abs[r] (the outer target) or more than
  // kGapRatio times the recurrence's: the FP32 convolution's rounding has
  // then become the larger part of the true residual, and only a new
  // correction from the FP64 residual (the outer step) reduces it further.
  long long check_every = 0;
  const double* check_abs = nullptr;
  bool adapt = false;              // mv32 solve that switches the convolution precision (MixedSwitch)
  int adapt_phase = 0;             // MixedSwitch phase
  double adapt_tau = 0;            // MixedSwitch phase 1 threshold
  char* stalled = nullptr;         // phase 0: per rhs, set when the FP32 start stalled
};

constexpr double kGapRatio = 4.0;  // |r_true|^2 > 4 |r_rec|^2: the gap dominates

// Precision of the convolution in an adaptive MIXED inner solve
// (SolveOpts::adapt), decided between rounds from the recurrence residuals.
//
// Phase 0 (the first inner solve): the FP32 convolution from the start,
// which is the whole solve for well-conditioned targets.  A right-hand side
// whose best residual does not halve within kStallStart iterations ends its
// inner solve with `stalled` set: on large, high-index targets QMR-CS with
// the FP32 convolution stays on a residual plateau that the FP64 solve
// leaves after a few thousand iterations, and a Krylov space built with the
// FP32 rounding does not recover when continued in FP64, so the outer step
// restarts it.
//
// Phase 1 (after a stall): the FP64 convolution until every running
// right-hand side is below tau (200 times its inner target: the rounding
// the FP32 convolution then adds to each Krylov vector scales with a
// residual that is already small), then the FP32 convolution in the same
// Krylov space.  If that stalls (no halving within kStallLate iterations)
// the solve continues, again in the same Krylov space, with the FP64
// convolution until the residual has fallen a hundredfold below the stall.
constexpr long long kStallStart = 256, kStallLate = 1024;

struct MixedSwitch {
  int phase = 0;
  bool mode32 = true;
  double tau = 0;            // phase 1: FP64 -> FP32 below this
  long long it32 = 0;        // iterations run with the FP32 convolution
  long long mark_it = -1;    // phase 1: start of the current FP32 window
  double mark = 0;
  std::vector<long long> rmark_it;  // phase 0: per rhs
  std::vector<double> rmark;
  MixedSwitch(int phase_, double tau_, int nrhs)
      : phase(phase_), mode32(phase_ == 0), tau(tau_), rmark_it(nrhs, -1), rmark(nrhs, 0) {}
  // Called after each round; phase 0 may end right-hand sides (returns true
  // when it changed a done flag in st).
  bool update(KrylovState* st, int nrhs, long long nr, long long poll, char* stalled) {
    bool changed = false;
    if (mode32) it32 += poll;
    if (phase == 0) {
      for (int r = 0; r < nrhs; r++) {
        if (st[r].done) continue;
        const double rel = std::sqrt(st[r].inprodR * st[r].residScale);
        if (rmark_it[r] < 0) {
          rmark_it[r] = nr;
          rmark[r] = rel;
        } else if (nr - rmark_it[r] >= kStallStart) {
          if (rel > 0.5 * rmark[r]) {
            st[r].done = 1;
            stalled[r] = 1;
            changed = true;
          } else {
            rmark_it[r] = nr;
            rmark[r] = rel;
          }
        }
      }
      return changed;
    }
    double worst = 0;
    for (int r = 0; r < nrhs; r++)
      if (!st[r].done) worst = std::max(worst, std::sqrt(st[r].inprodR * st[r].residScale));
    if (mode32) {
      if (mark_it < 0) {
        mark_it = nr;
        mark = worst;
      } else if (nr - mark_it >= kStallLate) {
        if (worst > 0.5 * mark) {
          mode32 = false;
          tau = 0.01 * worst;
        } else {
          mark_it = nr;
          mark = worst;
        }
      }
    } else if (worst < tau) {
      mode32 = true;
      mark_it = nr;
      mark = worst;
    }
    return false;
  }
};

// The FP64 check of a MIXED inner solve (SolveOpts::check_every): T = B - A x
// with the full FP64 matvec into `tmp`, |T|^2 into the outer state's `last`;
// right-hand sides that met the outer target or whose true residual is
// dominated by the FP32 rounding gap are marked done.  Returns true when
// every right-hand side is done.
bool check_gap(dda_ctx* c, int nrhs, double2* X, double2* B, double2* tmp, const SolveOpts& o) {
  Solve<double> sc(c, nrhs, c->st_outer);
  sc.mv(X, tmp, 0, sc.step(KOP_NONE));
  sc.vec(V_R_INIT, 0, {tmp, tmp, B}, sc.step(KOP_NORM));
  CK(cudaMemcpyAsync(c->sto_host, c->st_outer, nrhs * sizeof(KrylovState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  bool changed = false, all = true;
  for (int r = 0; r < nrhs; r++) {
    KrylovState& k = c->st_host[r];
    if (!k.done && !c->sto_host[r].done) {
      const double t = c->sto_host[r].last;
      if (t < o.check_abs[r] || t > kGapRatio * k.last || !(t == t)) {
        k.done = 1;
        changed = true;
      }
    }
    all = all && k.done;
  }
  if (changed)
    CK(cudaMemcpyAsync(c->st, c->st_host, nrhs * sizeof(KrylovState), cudaMemcpyHostToDevice, c->stream));
  return all;
}

// Runs one solve of `nrhs` right-hand sides already set up in the engine
// vectors (E = einc or B = b, S = start).  Per-rhs states end in c->st_host;
// the solution x is left in engine vector 4.
template <typename T>
void run_solve(dda_ctx* c, int solver, int nrhs, double eps, long long max_iter, const SolveOpts& o) {
  typedef typename C2<T>::t T2;
  NvtxRange range(sizeof(T) == 4 ? "dda solve fp32" : (o.mv32 || o.adapt) ? "dda inner solve" : "dda solve fp64");
  Engine<T>& e = eng<T>(c);
  Solve<T> sv(c, nrhs);
  sv.mv32 = o.mv32;
  T2 *E = e.vec[0], *B = e.vec[1], *S = e.vec[2];
  typename Solve<T>::Bufs b{e.vec[3], e.vec[4], e.vec[5], e.vec[6], e.vec[7], e.vec[8], e.vec[9]};
  // initial state
  for (int r = 0; r < nrhs; r++) {
    KrylovState& k = c->st_host[r];
    memset(&k, 0, sizeof(k));
    k.maxIter = max_iter > 0 ? max_iter : (1LL << 62);
    k.maxResIncrease = o.max_res_increase > 0 ? o.max_res_increase : kMaxResIncrease[solver];
    k.rateWin = o.rate_window;
    k.histCap = c->hist_cap;
    k.hist = c->hist + (size_t)r * c->hist_cap;
    if (o.skip && o.skip[r]) k.done = 1;
  }
  CK(cudaMemcpyAsync(c->st, c->st_host, nrhs * sizeof(KrylovState), cudaMemcpyHostToDevice, c->stream));
  sv.init_general(E, B, b.R, b.X, b.A, S, o.start, o.b_given);
  // epsB = eps^2 / residScale (DDA/IterativeSolverBase.cpp:44)
  CK(cudaMemcpyAsync(c->st_host, c->st, nrhs * sizeof(KrylovState), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int r = 0; r < nrhs; r++) {
    KrylovState& k = c->st_host[r];
    const double er = o.eps_rhs ? o.eps_rhs[r] : eps;
    k.epsB = er * er / k.residScale;
    if (k.done) continue;
    if (!std::isfinite(k.temp) || !std::isfinite(k.inprodR)) {  // NaN or Inf in Einc, sqrt(cc) or start
      k.done = 1;
      k.status = DDA_ERR_ARG;
    } else if (k.temp == 0) {  // b = 0: x = 0 is the solution
      k.done = 1;
    } else if (!(k.inprodR >= k.epsB)) {
      k.done = 1;  // already converged: no iteration
    }
  }
  CK(cudaMemcpyAsync(c->st, c->st_host, nrhs * sizeof(KrylovState), cudaMemcpyHostToDevice, c->stream));
  sv.solver_init(solver, b);
  long long nr = 0;
  // The host looks at the convergence flags every `poll` iterations.  The
  // first round (iterations 0..7 hold the solvers' first-iteration variants)
  // is launched kernel by kernel; the second round is captured into a CUDA
  // graph once and every later round replays it.  poll is even, so the
  // buffers the solvers rotate on the host are back in the captured order
  // after each round; all other kernel arguments are fixed pointers, and
  // the kernels read their scalars and done flags from the device state.
  const int poll = 8;
  const bool graphs = !(c->flags & DDA_FLAG_NO_GRAPHS);
  // graph of the current kernel sequence (index into c->round_graphs, which
  // may grow while this solve runs: a precision switch captures a second one)
  auto find_graph = [&](int key) -> int {
    for (size_t i = 0; i < c->round_graphs.size(); i++) {
      const auto& x = c->round_graphs[i];
      if (x.solver == solver && x.nrhs == nrhs && x.tsize == key) return (int)i;
    }
    return -1;
  };
  MixedSwitch ms(o.adapt_phase, o.adapt_tau, nrhs);
  if (o.adapt) sv.mv32 = ms.mode32;
  for (int round = 0;; round++) {
    if constexpr (std::is_same<T, double>::value) {
      if (!sv.mv32 && !c->e64_tuned) {  // first FP64-convolution round of a MIXED context
        c->e64_tuned = true;
        autotune<double>(c);
      }
    }
    if (!graphs || round == 0) {
      for (int k = 0; k < poll; k++) sv.iteration(solver, nr++, b);
    } else {
      const int gkey = (int)sizeof(T) + (sv.mv32 ? 100 : 0);  // kernel sequences differ per variant
      int gi = find_graph(gkey);
      if (gi < 0) {  // capture once per context, solver, batch and precision
        const long long l0 = c->launches;
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        try {
          for (int k = 0; k < poll; k++) sv.iteration(solver, nr + k, b);
        } catch (...) {
          cudaStreamEndCapture(c->stream, &graph);
          if (graph) cudaGraphDestroy(graph);
          throw;
        }
        CK(cudaStreamEndCapture(c->stream, &graph));
        cudaGraphExec_t g = nullptr;
        const cudaError_t rc = cudaGraphInstantiate(&g, graph, 0);
        cudaGraphDestroy(graph);
        CK(rc);
        c->round_graphs.push_back({solver, nrhs, gkey, g, c->launches - l0});
        gi = (int)c->round_graphs.size() - 1;
        c->launches = l0;
      }
      CK(cudaGraphLaunch(c->round_graphs[gi].g, c->stream));
      c->launches += c->round_graphs[gi].launches;
      nr += poll;
    }
    {
      NvtxRange wait("dda round: wait for the state");
      CK(cudaMemcpyAsync(c->st_host, c->st, nrhs * sizeof(KrylovState), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
    bool all = true;
    for (int r = 0; r < nrhs; r++) all = all && c->st_host[r].done;
    if (all) break;
    if (c->cancel.load()) {  // dda_cancel from another thread: stop between rounds
      for (int r = 0; r < nrhs; r++)
        if (!c->st_host[r].done) {
          c->st_host[r].done = 1;
          c->st_host[r].status = DDA_ERR_CANCELLED;
        }
      CK(cudaMemcpyAsync(c->st, c->st_host, nrhs * sizeof(KrylovState), cudaMemcpyHostToDevice, c->stream));
      break;
    }
    if constexpr (std::is_same<T, double>::value) {
      // the FP64 check only once the FP32 convolution has run (the gap is
      // its rounding carried along)
      // and only once some right-hand side's recurrence residual is within
      // a hundred times its target (earlier the gap cannot dominate)
      bool near = false;
      for (int r = 0; r < nrhs && !near; r++) {
        const KrylovState& k = c->st_host[r];
        near = !k.done && k.inprodR < 1e4 * k.epsB;
      }
      const bool gap_possible = (!o.adapt || ms.it32 > 0) && near;
      if (o.check_every > 0 && nr % o.check_every == 0 && gap_possible && check_gap(c, nrhs, b.X, B, S, o)) break;
      if (o.adapt) {
        if (ms.update(c->st_host, nrhs, nr, poll, o.stalled)) {
          CK(cudaMemcpyAsync(c->st, c->st_host, nrhs * sizeof(KrylovState), cudaMemcpyHostToDevice, c->stream));
          bool all_done = true;
          for (int r = 0; r < nrhs; r++) all_done = all_done && c->st_host[r].done;
          if (all_done) break;
        }
        sv.mv32 = ms.mode32;
      }
    }
  }
  if (b.X != e.vec[4])
    CK(cudaMemcpyAsync(e.vec[4], b.X, (size_t)nrhs * 3 * c->g.nvs * sizeof(T2), cudaMemcpyDeviceToDevice, c->stream));
  // P = sqrt(cc) x
  if (o.result) sv.vec(V_RESULT, 0, {e.io, e.vec[4]}, KrylovStep{KOP_NONE, 0, nullptr, {}});
}

// Mixed precision: inner solves of A e = r corrected by FP64 residuals
// r = b - A x until |r| < eps |b| in FP64.  Per-rhs totals are returned in
// out[] (iterations, refinements, status, best relative residual).
struct MixedOut {
  long long iterations = 0, refinements = 0;
  int status = 0;
  double rel = 0, res_scale = 0;
};

void run_mixed(dda_ctx* c, int solver, int nrhs, double eps, long long max_iter, bool start,
               std::vector<MixedOut>& out) {
  NvtxRange range("dda mixed refinement");
  Engine<double>& d = c->e64;
  Solve<double> sd(c, nrhs, c->st_outer);
  const size_t n = (size_t)nrhs * 3 * c->g.nvs;
  // E (incident field) and S (start) as for run_solve; the refined solution
  // and b live in xo, bo; the inner solves take their right-hand side r in
  // vector 1 and leave their solution in vector 4 (vectors 3..9 are theirs)
  double2 *E = d.vec[0], *R = d.vec[1], *S = d.vec[2], *A = d.vec[6], *X = d.xo, *B = d.bo;
  out.assign(nrhs, MixedOut());
  for (int r = 0; r < nrhs; r++) memset(&c->sto_host[r], 0, sizeof(KrylovState));
  CK(cudaMemcpyAsync(c->st_outer, c->sto_host, nrhs * sizeof(KrylovState), cudaMemcpyHostToDevice, c->stream));
  sd.vec(V_SETUP_PVEC, 0, {B, E}, sd.step(KOP_INIT_PVEC));  // b = sqrt(cc) Einc, |b|^2
  if (start) sd.vec(V_START_X, 0, {X, S}, KrylovStep{KOP_NONE, 0, nullptr, {}});
  else CK(cudaMemsetAsync(X, 0, n * sizeof(double2), c->stream));
  std::vector<char> done(nrhs, 0);
  std::vector<double> eps_in(nrhs, 1e-4), thr(nrhs, 0.0);
  // Each inner solve is an FP64 Krylov solve of A e = r (FP64 vectors,
  // scalars and dot products) whose matvec runs the convolution in FP32
  // (Solve::matvec_any).  It keeps one Krylov space for as long as that
  // helps: it aims at the final target and is checked against the FP64
  // residual every kCheckEvery iterations (check_gap).  It ends when the
  // FP64 residual meets the target, or when the residual the recurrences
  // track has fallen well below the true one: the FP32 convolution's
  // rounding, carried by every Krylov vector, then dominates, and the next
  // outer step removes it from a new FP64 residual.  Plateaus of the
  // recurrence (QMR-CS stagnates for hundreds of iterations on large,
  // high-index targets) do not end it.  A right-hand side whose FP64
  // residual does not halve over kOuterStall outer steps in a row leaves the
  // refinement with DDA_ERR_NOPROGRESS, and mixed_fallback finishes it with
  // the FP64 solver.
  const int max_outer = 60;
  const long long kCheckEvery = 64;
  const int kOuterStall = 2;
  std::vector<double> prev_rel(nrhs, 0.0);
  std::vector<int> stalls(nrhs, 0);
  std::vector<char> fp32_stalled(nrhs, 0);  // the FP32 start stalled (MixedSwitch phase 0)
  for (int outer = 0;; outer++) {
    // r = b - A x (full FP64 matvec); reduction n = |r|^2 -> last
    if (outer > 0 || start) sd.mv(X, A, 0, sd.step(KOP_NONE));
    else CK(cudaMemsetAsync(A, 0, n * sizeof(double2), c->stream));
    sd.vec(V_R_INIT, 0, {R, A, B}, sd.step(KOP_NORM));
    CK(cudaMemcpyAsync(c->sto_host, c->st_outer, nrhs * sizeof(KrylovState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    bool all = true;
    long long total_it = 0;
    for (int r = 0; r < nrhs; r++) {
      KrylovState& k = c->sto_host[r];
      const double rel = std::sqrt(k.last * k.residScale);
      out[r].rel = rel;
      out[r].res_scale = k.residScale;
      total_it = std::max(total_it, out[r].iterations);
      if (!done[r] && outer == 0 && !std::isfinite(k.temp)) { done[r] = 1; out[r].status = DDA_ERR_ARG; }
      if (!done[r] && outer == 0 && k.temp == 0) done[r] = 1;  // b = 0: x = 0
      if (!done[r] && !(rel == rel)) { done[r] = 1; out[r].status = DDA_ERR_BREAKDOWN; }
      if (!done[r] && (rel < eps || out[r].status != 0)) done[r] = 1;
      if (!done[r] && outer > 0) {
        stalls[r] = rel > 0.5 * prev_rel[r] ? stalls[r] + 1 : 0;
        if (stalls[r] >= kOuterStall) { done[r] = 1; out[r].status = DDA_ERR_NOPROGRESS; }
      }
      prev_rel[r] = rel;
      if (!done[r] && outer >= max_outer) { done[r] = 1; out[r].status = DDA_ERR_NOPROGRESS; }
      if (!done[r] && max_iter > 0 && out[r].iterations >= max_iter) { done[r] = 1; out[r].status = DDA_ERR_MAXITER; }
      if (!done[r] && c->cancel.load()) { done[r] = 1; out[r].status = DDA_ERR_CANCELLED; }
      k.done = done[r];
      // the FP64 recurrences can follow the inner system to the final target
      // in one go; the FP32 convolution then leaves a residual of about its
      // own rounding times the condition number, which the next outer step
      // removes
      eps_in[r] = std::min(0.1, std::max(1e-7, 0.5 * eps / rel));
      thr[r] = 0.81 * eps * eps / k.residScale;  // (0.9 eps |b|)^2
      all = all && done[r];
    }
    if (all) break;
    CK(cudaMemcpyAsync(c->st_outer, c->sto_host, nrhs * sizeof(KrylovState), cudaMemcpyHostToDevice, c->stream));
    SolveOpts o;
    o.b_given = true;
    o.eps_rhs = eps_in.data();
    o.skip = done.data();
    o.result = false;
    o.mv32 = true;
    o.adapt = true;
    o.adapt_phase = 0;
    double eps_max = 0;
    for (int r = 0; r < nrhs; r++)
      if (!done[r]) {
        if (fp32_stalled[r]) o.adapt_phase = 1;
        eps_max = std::max(eps_max, eps_in[r]);
      }
    o.adapt_tau = 200 * eps_max;
    std::vector<char> stalled_now(nrhs, 0);
    o.stalled = stalled_now.data();
    o.check_every = kCheckEvery;
    o.check_abs = thr.data();
    run_solve<double>(c, solver, nrhs, 0.0, max_iter > 0 ? max_iter - total_it : 0, o);
    for (int r = 0; r < nrhs; r++)
      if (stalled_now[r]) fp32_stalled[r] = 1;
    for (int r = 0; r < nrhs; r++) {
      if (done[r]) continue;
      out[r].iterations += c->st_host[r].count;
      out[r].refinements++;
      if (c->st_host[r].status == DDA_ERR_CANCELLED) out[r].status = DDA_ERR_CANCELLED;
      // an inner solve that stopped early (stagnation, breakdown, its share
      // of max_iter) still contributes its correction; the outer FP64
      // residual decides
    }
    // x += e for the rhs still running
    k_accum<double2><<<dim3(c->nparts_vec, nrhs), 256, 0, c->stream>>>(X, d.vec[4], c->st_outer, 3LL * c->g.nvs);
    CK(cudaGetLastError());
    c->launches++;
  }
  sd.vec(V_RESULT, 0, {d.io, X}, KrylovStep{KOP_NONE, 0, nullptr, {}});
}

}  // namespace

// ================================================================ C ABI ===
extern "C" {

const char* dda_last_error(const dda_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int dda_create(const dda_problem* p, int precision, dda_ctx** out) {
  NvtxRange range("dda create");
  if (!p || !out) {
    g_create_error = "null argument";
    return DDA_ERR_ARG;
  }
  *out = nullptr;
  std::unique_ptr<dda_ctx> c(new dda_ctx);
  c->device = p->device;
  int rc = guard(nullptr, [&]() -> int {
    if (p->nv == 0 || !p->positions) throw DdaError(DDA_ERR_ARG, "empty geometry");
    if (precision < DDA_PREC_FP64 || precision > DDA_PREC_MIXED) throw DdaError(DDA_ERR_ARG, "bad precision");
    if (p->nmat == 0 || p->nmat > 256) throw DdaError(DDA_ERR_ARG, "nmat must be 1..256");
    if (p->max_rhs < 1) throw DdaError(DDA_ERR_ARG, "max_rhs must be >= 1");
    if (!(p->grid_unit > 0) || !(p->kd > 0)) throw DdaError(DDA_ERR_ARG, "grid_unit and kd must be positive");
    for (int a = 0; a < 3; a++) {
      if (p->box[a] == 0 || p->grid[a] % 2 != 0 || p->grid[a] < 2 * p->box[a])
        throw DdaError(DDA_ERR_ARG, "grid must be even and at least twice the box");
    }
    // one grid line must fit the register tiles of a CTA (FP64 limits apply
    // to the D-matrix setup in every precision)
    const uint32_t lim = 4096;
    if (p->box[0] >= 65536 || p->grid[0] > lim || p->grid[1] > lim || p->grid[2] > lim)
      throw DdaError(DDA_ERR_UNSUPPORTED, "FFT grid edge above " + std::to_string(lim));
    CK(cudaSetDevice(p->device));
    g_dalloc_bytes = 0;
    c->precision = precision;
    c->max_rhs = p->max_rhs;
    c->flags = p->flags;
    c->kd = p->kd;
    c->grid_unit = p->grid_unit;
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    g_alloc_stream = c->stream;
    MvGeom& g = c->g;
    g.Gx = p->grid[0]; g.Gy = p->grid[1]; g.Gz = p->grid[2];
    g.bx = p->box[0]; g.by = p->box[1]; g.bz = p->box[2];
    g.nv = (int)p->nv;
    g.nvs = (int)((p->nv + 15) / 16 * 16);  // DDA/DDAParams.cpp:113
    g.nlines = g.by * g.bz;
    g.nmat = (int)p->nmat;
    g.pitchx = g.Gx + 1;
    g.tl = 0;  // per engine (Engine::tl), set in the copy each launch takes
    // geometry tables: dipoles sorted by grid line (y + by z), stable
    const uint32_t nv = p->nv;
    std::vector<uint32_t> line(nv), cnt(g.nlines + 1, 0);
    for (uint32_t i = 0; i < nv; i++) {
      const uint32_t x = p->positions[3 * i], y = p->positions[3 * i + 1], z = p->positions[3 * i + 2];
      if (x >= p->box[0] || y >= p->box[1] || z >= p->box[2]) throw DdaError(DDA_ERR_ARG, "dipole outside the box");
      const uint8_t m = p->materials ? p->materials[i] : 0;
      if (m >= p->nmat) throw DdaError(DDA_ERR_ARG, "material index out of range");
      line[i] = y + (uint32_t)g.by * z;
      cnt[line[i] + 1]++;
    }
    for (int l = 0; l < g.nlines; l++) cnt[l + 1] += cnt[l];
    std::vector<uint32_t> off(cnt), perm(nv), dip(nv);
    std::vector<uint8_t> matx(nv);
    bool ident = true;
    std::vector<std::vector<char>> seen;  // duplicate check per line via x bitmap
    std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
    for (uint32_t i = 0; i < nv; i++) {
      const uint32_t j = fill[line[i]]++;
      perm[j] = i;
      if (j != i) ident = false;
      const uint8_t m = p->materials ? p->materials[i] : 0;
      dip[j] = p->positions[3 * i] | ((uint32_t)m << 16);
      matx[i] = m;
    }
    dmalloc((void**)&c->line_off, off.size() * sizeof(uint32_t));
    CK(cudaMemcpyAsync(c->line_off, off.data(), off.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    dmalloc((void**)&c->dip, nv * sizeof(uint32_t));
    CK(cudaMemcpyAsync(c->dip, dip.data(), nv * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    if (!ident) {
      dmalloc((void**)&c->perm, nv * sizeof(uint32_t));
      CK(cudaMemcpyAsync(c->perm, perm.data(), nv * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
    }
    dmalloc((void**)&c->mat_ext, nv);
    CK(cudaMemcpyAsync(c->mat_ext, matx.data(), nv, cudaMemcpyHostToDevice, c->stream));
    c->px.create(g.Gx);
    c->py.create(g.Gy);
    c->pz.create(g.Gz);
    c->planned = has_tuned_plan(g.Gx) && has_tuned_plan(g.Gy) && has_tuned_plan(g.Gz) &&
                 !(c->flags & DDA_FLAG_RUNTIME_PLANS);
    c->mx.create(g.Gx, c->planned ? tuned_radices(g.Gx) : std::vector<int>());
    c->my.create(g.Gy, c->planned ? tuned_radices(g.Gy) : std::vector<int>());
    c->mz.create(g.Gz, c->planned ? tuned_radices(g.Gz) : std::vector<int>());
    g.fx = c->mx.freq;
    g.fy = c->my.freq;
    g.fz = c->mz.freq;
    if (precision != DDA_PREC_FP32) setup_engine<double>(c.get());
    if (precision != DDA_PREC_FP64) setup_engine<float>(c.get());
    // reduction slots
    c->nparts_mv = 3 * std::max(c->e32.on ? ntiles(c.get(), c->e32.tl) : 0,
                                c->e64.on ? ntiles(c.get(), c->e64.tl) : 0);
    c->nparts_vec = vec_parts(c.get());
    const int nparts = std::max(c->nparts_mv, c->nparts_vec);
    dmalloc((void**)&c->parts, (size_t)c->max_rhs * nparts * sizeof(RedSums));
    dmalloc((void**)&c->tickets, c->max_rhs * sizeof(unsigned));
    CK(cudaMemsetAsync(c->tickets, 0, c->max_rhs * sizeof(unsigned), c->stream));
    dmalloc((void**)&c->st, c->max_rhs * sizeof(KrylovState));
    CK(cudaMemsetAsync(c->st, 0, c->max_rhs * sizeof(KrylovState), c->stream));
    c->st_host = new KrylovState[c->max_rhs];
    dmalloc((void**)&c->st_outer, c->max_rhs * sizeof(KrylovState));
    CK(cudaMemsetAsync(c->st_outer, 0, c->max_rhs * sizeof(KrylovState), c->stream));
    c->sto_host = new KrylovState[c->max_rhs];
    c->hist_cap = 100000;
    dmalloc((void**)&c->hist, (size_t)c->max_rhs * c->hist_cap * sizeof(double));
    c->cc_host.assign((size_t)c->max_rhs * g.nmat * 3, 0);
    c->cc_set.assign(c->max_rhs, 0);
    if (p->dmatrix) upload_dmatrix(c.get(), p->dmatrix);
    else build_dmatrix(c.get());
    if (!(c->flags & DDA_FLAG_NO_AUTOTUNE)) {
      if (c->e32.on) autotune<float>(c.get());
      // MIXED runs its FP64 engine for a few outer residuals and checks and,
      // for targets whose FP32 convolution stalls, the FP64 phases of its
      // inner solves: tuned on the first such phase (run_solve), which many
      // targets never reach, instead of here.  The shapes never change the
      // arithmetic.
      if (c->e64.on && precision == DDA_PREC_MIXED) c->e64_tuned = false;
      else if (c->e64.on) autotune<double>(c.get());
    }
    CK(cudaStreamSynchronize(c->stream));
    c->dev_bytes = g_dalloc_bytes;
    return DDA_OK;
  });
  if (rc != DDA_OK) {
    c->release();
    return rc;
  }
  *out = c.release();
  return DDA_OK;
}

int dda_destroy(dda_ctx* ctx) {
  if (!ctx) return DDA_OK;
  ctx->release();
  delete ctx;
  return DDA_OK;
}

int64_t dda_vec_stride(const dda_ctx* ctx) { return ctx ? ctx->g.nvs : 0; }

int dda_set_cc(dda_ctx* ctx, int rhs, const double* cc_sqrt) {
  if (!ctx) return DDA_ERR_ARG;
  return guard(ctx, [&]() -> int {
    if (rhs < 0 || rhs >= ctx->max_rhs || !cc_sqrt) throw DdaError(DDA_ERR_ARG, "bad rhs index or null cc_sqrt");
    const int n = ctx->g.nmat * 3;
    for (int i = 0; i < 2 * n; i++)
      if (!std::isfinite(cc_sqrt[i])) throw DdaError(DDA_ERR_ARG, "couple constants are not finite");
    for (int i = 0; i < n; i++)
      ctx->cc_host[(size_t)rhs * n + i] = std::complex<double>(cc_sqrt[2 * i], cc_sqrt[2 * i + 1]);
    ctx->cc_set[rhs] = 1;
    upload_cc<float>(ctx);
    upload_cc<double>(ctx);
    return DDA_OK;
  });
}

int dda_matvec(dda_ctx* ctx, const void* d_arg, void* d_res, int conj, int nrhs, int precision,
               void* stream) {
  if (!ctx) return DDA_ERR_ARG;
  return guard(ctx, [&]() -> int {
    if (nrhs < 1 || nrhs > ctx->max_rhs || !d_arg || !d_res) throw DdaError(DDA_ERR_ARG, "bad matvec arguments");
    for (int r = 0; r < nrhs; r++)
      if (!ctx->cc_set[r]) throw DdaError(DDA_ERR_ARG, "couple constants not set (dda_set_cc)");
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    if (precision == DDA_PREC_FP64) {
      if (!ctx->e64.on) throw DdaError(DDA_ERR_ARG, "context has no FP64 engine");
      matvec<double>(ctx, (const double2*)d_arg, (double2*)d_res, conj, nrhs, s, nullptr, KrylovStep{KOP_NONE, 0, nullptr, {}});
    } else if (precision == DDA_PREC_FP32) {
      if (!ctx->e32.on) throw DdaError(DDA_ERR_ARG, "context has no FP32 engine");
      matvec<float>(ctx, (const float2*)d_arg, (float2*)d_res, conj, nrhs, s, nullptr, KrylovStep{KOP_NONE, 0, nullptr, {}});
    } else {
      throw DdaError(DDA_ERR_ARG, "precision must be DDA_PREC_FP64 or DDA_PREC_FP32");
    }
    return DDA_OK;
  });
}

}  // extern "C"

namespace {
// Stage timing for dda_profile_matvec: the three passes of matvec<T> with an
// event between them, on vectors the context owns.
template <typename T> void profile_t(dda_ctx* c, int nrhs, int reps, double* ms) {
  typedef typename C2<T>::t T2;
  Engine<T>& e = eng<T>(c);
  MvGeom g = c->g;
  g.tl = e.tl;
  const FftPlanDev px = c->mx.dev<T>();
  cudaStream_t s = c->stream;
  cudaEvent_t ev[4];
  for (auto& x : ev) CK(cudaEventCreate(&x));
  double acc[3] = {0, 0, 0};
  const T2* arg = e.vec[0];
  T2* res = e.io;
  KrylovStep none{KOP_NONE, 0, nullptr, {}};
  none.red = red_target(c, 3 * ntiles(c, e.tl));
  for (int r = 0; r <= reps; r++) {
    dim3 gx(ntiles(c, e.tl), 3, nrhs);
    CK(cudaEventRecord(ev[0], s));
    e.k.xfwd<<<gx, kNtX, e.smem_x, s>>>(arg, e.xhat, c->line_off, c->dip, c->perm, e.ccs, 0, g, px, nullptr, 0,
                                        XPre{});
    CK(cudaEventRecord(ev[1], s));
    launch_yz<T>(c, nrhs, s, nullptr, 0);
    CK(cudaEventRecord(ev[2], s));
    e.k.xinv<<<gx, kNtX, e.smem_x, s>>>(arg, res, e.xhat, c->line_off, c->dip, c->perm, e.ccs, 0, g, px, nullptr, none,
                                        0);
    CK(cudaEventRecord(ev[3], s));
    CK(cudaEventSynchronize(ev[3]));
    if (r == 0) continue;  // warm-up
    for (int k = 0; k < 3; k++) {
      float t;
      CK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      acc[k] += t;
    }
  }
  for (auto& x : ev) cudaEventDestroy(x);
  for (int k = 0; k < 3; k++) ms[k] = acc[k] / reps;
  ms[3] = ms[0] + ms[1] + ms[2];
}

// Host FP64 vectors and the FP32 engine: the FP64 data crosses the bus as it
// is and is rounded (to nearest, as a host cast would) on the device.  The
// FP64 copy is staged in two solver workspace vectors, which hold nothing
// before a solve starts or after it ends and of which each holds half of
// `n` FP64 complex values (n <= max_rhs 3 nvs, even).  With the input from
// pinned host memory the copies run at full bus speed and never block the
// host.
struct HostStage {
  double2* part[2];
  size_t len[2];
  void* temp = nullptr;
};

HostStage host_stage(dda_ctx* c, size_t n) {
  HostStage h;
  h.len[0] = n / 2;
  h.len[1] = n - n / 2;
  Engine<float>& e = c->e32;
  if (e.vec[8] && e.vec[9]) {
    h.part[0] = reinterpret_cast<double2*>(e.vec[8]);
    h.part[1] = reinterpret_cast<double2*>(e.vec[9]);
  } else {
    CK(cudaMallocAsync(&h.temp, n * sizeof(double2), c->stream));
    h.part[0] = static_cast<double2*>(h.temp);
    h.part[1] = h.part[0] + h.len[0];
  }
  return h;
}

void host_stage_release(dda_ctx* c, HostStage& h) {
  if (h.temp) CK(cudaFreeAsync(h.temp, c->stream));
  h.temp = nullptr;
}

template <typename T>
void host_to_engine(dda_ctx* c, const double* src, typename C2<T>::t* dst, size_t n) {
  if constexpr (std::is_same<T, double>::value) {
    CK(cudaMemcpyAsync(dst, src, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  } else {
    HostStage h = host_stage(c, n);
    size_t off = 0;
    for (int k = 0; k < 2; k++) {
      CK(cudaMemcpyAsync(h.part[k], src + 2 * off, h.len[k] * sizeof(double2), cudaMemcpyHostToDevice,
                         c->stream));
      k_convert<double2, float2><<<592, 256, 0, c->stream>>>(h.part[k], dst + off, (long long)h.len[k]);
      CK(cudaGetLastError());
      c->launches++;
      off += h.len[k];
    }
    host_stage_release(c, h);
  }
}
template <typename T>
void engine_to_host(dda_ctx* c, const typename C2<T>::t* src, double* dst, size_t n) {
  if constexpr (std::is_same<T, double>::value) {
    CK(cudaMemcpyAsync(dst, src, n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  } else {
    HostStage h = host_stage(c, n);
    size_t off = 0;
    for (int k = 0; k < 2; k++) {
      k_convert<float2, double2><<<592, 256, 0, c->stream>>>(src + off, h.part[k], (long long)h.len[k]);
      CK(cudaGetLastError());
      c->launches++;
      CK(cudaMemcpyAsync(dst + 2 * off, h.part[k], h.len[k] * sizeof(double2), cudaMemcpyDeviceToHost,
                         c->stream));
      off += h.len[k];
    }
    host_stage_release(c, h);
  }
  CK(cudaStreamSynchronize(c->stream));
}

template <typename T>
void matvec_host_t(dda_ctx* c, const double* arg, double* res, int conj, int nrhs) {
  Engine<T>& e = eng<T>(c);
  const size_t n = (size_t)nrhs * 3 * c->g.nvs;
  host_to_engine<T>(c, arg, e.vec[0], n);
  matvec<T>(c, e.vec[0], e.io, conj, nrhs, c->stream, nullptr, KrylovStep{KOP_NONE, 0, nullptr, {}});
  engine_to_host<T>(c, e.io, res, n);
}

int collect_stats(dda_ctx* c, int nrhs, double* history, long long history_cap, dda_stats* stats);

template <typename T>
int solve_t(dda_ctx* c, int solver, int nrhs, const double* einc, double eps, long long max_iter,
            const double* start, double* pol_out, double* history, long long history_cap,
            dda_stats* stats) {
  Engine<T>& e = eng<T>(c);
  const size_t n = (size_t)nrhs * 3 * c->g.nvs;
  host_to_engine<T>(c, einc, e.vec[0], n);
  if (start) host_to_engine<T>(c, start, e.vec[2], n);
  SolveOpts o;
  o.start = start != nullptr;
  run_solve<T>(c, solver, nrhs, eps, max_iter, o);
  if (pol_out) engine_to_host<T>(c, e.io, pol_out, n);
  CK(cudaStreamSynchronize(c->stream));
  return collect_stats(c, nrhs, history, history_cap, stats);
}

// FP32 context, single-precision host arrays: the fields cross the bus as
// they are (complex float, the engine's own layout), with no conversion.
int solve_f32_host(dda_ctx* c, int solver, int nrhs, const float* einc, double eps, long long max_iter,
                   const float* start, float* pol_out, double* history, long long history_cap, dda_stats* stats) {
  Engine<float>& e = c->e32;
  const size_t bytes = (size_t)nrhs * 3 * c->g.nvs * sizeof(float2);
  CK(cudaMemcpyAsync(e.vec[0], einc, bytes, cudaMemcpyHostToDevice, c->stream));
  if (start) CK(cudaMemcpyAsync(e.vec[2], start, bytes, cudaMemcpyHostToDevice, c->stream));
  SolveOpts o;
  o.start = start != nullptr;
  run_solve<float>(c, solver, nrhs, eps, max_iter, o);
  if (pol_out) CK(cudaMemcpyAsync(pol_out, e.io, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return collect_stats(c, nrhs, history, history_cap, stats);
}

template <typename T>
int solve_device_t(dda_ctx* c, int solver, int nrhs, const void* einc, double eps, long long max_iter,
                   const void* start, void* pol, dda_stats* stats) {
  typedef typename C2<T>::t T2;
  Engine<T>& e = eng<T>(c);
  const size_t bytes = (size_t)nrhs * 3 * c->g.nvs * sizeof(T2);
  CK(cudaMemcpyAsync(e.vec[0], einc, bytes, cudaMemcpyDeviceToDevice, c->stream));
  if (start) CK(cudaMemcpyAsync(e.vec[2], start, bytes, cudaMemcpyDeviceToDevice, c->stream));
  SolveOpts o;
  o.start = start != nullptr;
  run_solve<T>(c, solver, nrhs, eps, max_iter, o);
  CK(cudaMemcpyAsync(pol, e.io, bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return collect_stats(c, nrhs, nullptr, 0, stats);
}

// Right-hand sides the mixed refinement could not finish (no progress,
// breakdown) are solved again with the FP64 solver, starting from the
// refined polarisations (e64.io); the others keep their result.  E (e64
// vector 0) still holds the incident fields.
void mixed_fallback(dda_ctx* c, int solver, int nrhs, double eps, long long max_iter, std::vector<MixedOut>& mo) {
  std::vector<char> skip(nrhs, 1);
  bool any = false;
  for (int r = 0; r < nrhs; r++)
    if (mo[r].status == DDA_ERR_NOPROGRESS || mo[r].status == DDA_ERR_BREAKDOWN) {
      skip[r] = 0;
      any = true;
    }
  if (!any) return;
  Engine<double>& d = c->e64;
  const size_t len = (size_t)3 * c->g.nvs;
  double2* S = d.vec[2];
  CK(cudaMemcpyAsync(S, d.io, nrhs * len * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
  SolveOpts o;
  o.start = true;
  o.skip = skip.data();
  long long used = 0;
  for (int r = 0; r < nrhs; r++) used = std::max(used, mo[r].iterations);
  run_solve<double>(c, solver, nrhs, eps, max_iter > 0 ? std::max(1LL, max_iter - used) : 0, o);
  for (int r = 0; r < nrhs; r++) {
    if (skip[r]) {  // the FP64 pass wrote io for every rhs: put the refined result back
      CK(cudaMemcpyAsync(d.io + r * len, S + r * len, len * sizeof(double2), cudaMemcpyDeviceToDevice, c->stream));
      continue;
    }
    const KrylovState& k = c->st_host[r];
    mo[r].iterations += k.count;
    mo[r].status = k.status;
    mo[r].rel = std::sqrt(k.inprodR * k.residScale);
  }
}

int collect_mixed(dda_ctx* c, const std::vector<MixedOut>& mo, double* history, long long history_cap,
                  dda_stats* stats) {
  int rc = DDA_OK;
  const int nrhs = (int)mo.size();
  for (int r = 0; r < nrhs; r++) {
    if (stats) {
      stats[r].iterations = mo[r].iterations;
      stats[r].matvecs = 0;
      stats[r].refinements = mo[r].refinements;
      stats[r].rel_residual = mo[r].rel;
      stats[r].res_scale = mo[r].res_scale;
      stats[r].status = mo[r].status;
    }
    if (history && history_cap > 0) {  // residual history of the last inner solve
      const long long m = std::min<long long>(std::min(history_cap, c->hist_cap), c->st_host[r].count);
      if (m > 0)
        CK(cudaMemcpyAsync(history + (size_t)r * history_cap, c->hist + (size_t)r * c->hist_cap,
                           m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (mo[r].status != 0 && rc == DDA_OK) rc = mo[r].status;
  }
  CK(cudaStreamSynchronize(c->stream));  // history copies done
  if (rc != DDA_OK)
    c->err = rc == DDA_ERR_MAXITER ? "Too many iterations"
           : rc == DDA_ERR_CANCELLED ? "cancelled"
           : rc == DDA_ERR_ARG ? "right-hand side or start value is not finite"
                               : "refinement did not converge";
  return rc;
}

int solve_mixed_host(dda_ctx* c, int solver, int nrhs, const double* einc, double eps, long long max_iter,
                     const double* start, double* pol_out, double* history, long long history_cap,
                     dda_stats* stats) {
  const size_t n = (size_t)nrhs * 3 * c->g.nvs;
  CK(cudaMemcpyAsync(c->e64.vec[0], einc, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  if (start) CK(cudaMemcpyAsync(c->e64.vec[2], start, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
  std::vector<MixedOut> mo;
  run_mixed(c, solver, nrhs, eps, max_iter, start != nullptr, mo);
  mixed_fallback(c, solver, nrhs, eps, max_iter, mo);
  if (pol_out) CK(cudaMemcpyAsync(pol_out, c->e64.io, n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return collect_mixed(c, mo, history, history_cap, stats);
}

int solve_mixed_device(dda_ctx* c, int solver, int nrhs, const void* einc, double eps, long long max_iter,
                       const void* start, void* pol, dda_stats* stats) {
  const size_t bytes = (size_t)nrhs * 3 * c->g.nvs * sizeof(double2);
  CK(cudaMemcpyAsync(c->e64.vec[0], einc, bytes, cudaMemcpyDeviceToDevice, c->stream));
  if (start) CK(cudaMemcpyAsync(c->e64.vec[2], start, bytes, cudaMemcpyDeviceToDevice, c->stream));
  std::vector<MixedOut> mo;
  run_mixed(c, solver, nrhs, eps, max_iter, start != nullptr, mo);
  mixed_fallback(c, solver, nrhs, eps, max_iter, mo);
  CK(cudaMemcpyAsync(pol, c->e64.io, bytes, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return collect_mixed(c, mo, nullptr, 0, stats);
}

int collect_stats(dda_ctx* c, int nrhs, double* history, long long history_cap, dda_stats* stats) {
  int rc = DDA_OK;
  for (int r = 0; r < nrhs; r++) {
    const KrylovState& k = c->st_host[r];
    if (stats) {
      stats[r].iterations = k.count;
      stats[r].matvecs = 0;
      stats[r].refinements = 0;
      stats[r].rel_residual = std::sqrt(k.inprodR * k.residScale);
      stats[r].res_scale = k.residScale;
      stats[r].status = k.status;
    }
    if (history && history_cap > 0) {
      const long long m = std::min<long long>(std::min(history_cap, c->hist_cap), k.count);
      if (m > 0)
        CK(cudaMemcpyAsync(history + (size_t)r * history_cap, c->hist + (size_t)r * c->hist_cap,
                           m * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (k.status != 0 && rc == DDA_OK) rc = k.status;
  }
  CK(cudaStreamSynchronize(c->stream));  // history copies done
  if (rc != DDA_OK) {
    static const char* msg[] = {"", "right-hand side or start value is not finite", "", "", "",
                                "Krylov breakdown", "Too many iterations", "Too many iterations w/o increase",
                                "cancelled"};
    c->err = (rc <= -5 && rc >= -8) || rc == -1 ? msg[-rc] : "solver failed";
  }
  return rc;
}
}  // namespace

extern "C" {

int dda_matvec_host(dda_ctx* ctx, const double* arg, double* res, int conj, int nrhs) {
  if (!ctx) return DDA_ERR_ARG;
  return guard(ctx, [&]() -> int {
    if (nrhs < 1 || nrhs > ctx->max_rhs || !arg || !res) throw DdaError(DDA_ERR_ARG, "bad matvec arguments");
    for (int r = 0; r < nrhs; r++)
      if (!ctx->cc_set[r]) throw DdaError(DDA_ERR_ARG, "couple constants not set (dda_set_cc)");
    if (ctx->e64.on) matvec_host_t<double>(ctx, arg, res, conj, nrhs);
    else matvec_host_t<float>(ctx, arg, res, conj, nrhs);
    return DDA_OK;
  });
}

int dda_solve(dda_ctx* ctx, int solver, int nrhs, const double* einc, double eps, int64_t max_iter,
              const double* start, double* pol_out, double* history, int64_t history_cap,
              dda_stats* stats) {
  if (!ctx) return DDA_ERR_ARG;
  const int rc = guard(ctx, [&]() -> int {
    if (solver < 0 || solver > 3) throw DdaError(DDA_ERR_ARG, "unknown solver");
    if (nrhs < 1 || nrhs > ctx->max_rhs || !einc) throw DdaError(DDA_ERR_ARG, "bad solve arguments");
    if (!(eps > 0)) throw DdaError(DDA_ERR_ARG, "eps must be positive");
    for (int r = 0; r < nrhs; r++)
      if (!ctx->cc_set[r]) throw DdaError(DDA_ERR_ARG, "couple constants not set (dda_set_cc)");
    if (ctx->precision == DDA_PREC_FP32)
      return solve_t<float>(ctx, solver, nrhs, einc, eps, max_iter, start, pol_out, history, history_cap, stats);
    if (ctx->precision == DDA_PREC_MIXED)
      return solve_mixed_host(ctx, solver, nrhs, einc, eps, max_iter, start, pol_out, history, history_cap, stats);
    return solve_t<double>(ctx, solver, nrhs, einc, eps, max_iter, start, pol_out, history, history_cap, stats);
  });
  ctx->cancel.store(0);
  return rc;
}

int dda_solve_f32(dda_ctx* ctx, int solver, int nrhs, const float* einc, double eps, int64_t max_iter,
                  const float* start, float* pol_out, double* history, int64_t history_cap, dda_stats* stats) {
  if (!ctx) return DDA_ERR_ARG;
  if (ctx->precision != DDA_PREC_FP32) {
    // FP64 and MIXED contexts: widen on the host (exact) and solve as
    // dda_solve (which also rejects bad arguments: einc NULL then)
    const bool ok = einc && nrhs >= 1 && nrhs <= ctx->max_rhs;
    const size_t n = ok ? (size_t)nrhs * 3 * ctx->g.nvs * 2 : 0;
    std::vector<double> e(ok ? einc : nullptr, ok ? einc + n : nullptr), s, p(pol_out ? n : 0);
    if (ok && start) s.assign(start, start + n);
    const int rc = dda_solve(ctx, solver, nrhs, ok ? e.data() : nullptr, eps, max_iter,
                             ok && start ? s.data() : nullptr, pol_out ? p.data() : nullptr, history, history_cap,
                             stats);
    if (pol_out)
      for (size_t i = 0; i < n; i++) pol_out[i] = (float)p[i];
    return rc;
  }
  const int rc = guard(ctx, [&]() -> int {
    if (solver < 0 || solver > 3) throw DdaError(DDA_ERR_ARG, "unknown solver");
    if (nrhs < 1 || nrhs > ctx->max_rhs || !einc) throw DdaError(DDA_ERR_ARG, "bad solve arguments");
    if (!(eps > 0)) throw DdaError(DDA_ERR_ARG, "eps must be positive");
    for (int r = 0; r < nrhs; r++)
      if (!ctx->cc_set[r]) throw DdaError(DDA_ERR_ARG, "couple constants not set (dda_set_cc)");
    return solve_f32_host(ctx, solver, nrhs, einc, eps, max_iter, start, pol_out, history, history_cap, stats);
  });
  ctx->cancel.store(0);
  return rc;
}

int dda_solve_device(dda_ctx* ctx, int solver, int nrhs, const void* d_einc, double eps, int64_t max_iter,
                     const void* d_start, void* d_pol, dda_stats* stats) {
  if (!ctx) return DDA_ERR_ARG;
  const int rc = guard(ctx, [&]() -> int {
    if (solver < 0 || solver > 3) throw DdaError(DDA_ERR_ARG, "unknown solver");
    if (nrhs < 1 || nrhs > ctx->max_rhs || !d_einc || !d_pol) throw DdaError(DDA_ERR_ARG, "bad solve arguments");
    if (!(eps > 0)) throw DdaError(DDA_ERR_ARG, "eps must be positive");
    for (int r = 0; r < nrhs; r++)
      if (!ctx->cc_set[r]) throw DdaError(DDA_ERR_ARG, "couple constants not set (dda_set_cc)");
    if (ctx->precision == DDA_PREC_FP64)
      return solve_device_t<double>(ctx, solver, nrhs, d_einc, eps, max_iter, d_start, d_pol, stats);
    if (ctx->precision == DDA_PREC_MIXED)
      return solve_mixed_device(ctx, solver, nrhs, d_einc, eps, max_iter, d_start, d_pol, stats);
    return solve_device_t<float>(ctx, solver, nrhs, d_einc, eps, max_iter, d_start, d_pol, stats);
  });
  ctx->cancel.store(0);
  return rc;
}

int dda_cancel(dda_ctx* ctx) {
  if (!ctx) return DDA_ERR_ARG;
  ctx->cancel.store(1);
  return DDA_OK;
}

void* dda_stream(dda_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t dda_launch_count(const dda_ctx* ctx) { return ctx ? ctx->launches : 0; }

int dda_choose_grid(const uint32_t* box, int policy, uint32_t* grid) {
  if (!box || !grid || policy < DDA_GRID_REFERENCE || policy > DDA_GRID_TUNED) return DDA_ERR_ARG;
  for (int a = 0; a < 3; a++) grid[a] = dda_fft_fit(2 * box[a], 0, 1);  // DDA/DDAParams.cpp:290-335
  if (policy == DDA_GRID_REFERENCE) return DDA_OK;
  auto tuned_ceil = [](uint32_t x) -> uint32_t {
    uint32_t best = 0;
#define C(N) if ((uint32_t)N >= x && (best == 0 || (uint32_t)N < best)) best = N;
    DDA_TUNED_LENGTHS(C)
#undef C
    return best;
  };
  const uint32_t gx = tuned_ceil(2 * box[0]), gyz = tuned_ceil(2 * std::max(box[1], box[2]));
  if (!gx || !gyz) return DDA_OK;
  const double ref = (double)grid[0] * grid[1] * grid[2], tun = (double)gx * gyz * gyz;
  if (tun > 2.0 * ref) return DDA_OK;  // padding would cost more than the plans gain
  grid[0] = gx;
  grid[1] = grid[2] = gyz;
  return DDA_OK;
}

// Upper bound of the device memory dda_create takes for `p`: the buffers the
// context keeps (resident) and, in addition while it is built, the FP64 grid
// of the D-matrix generation (peak).  Mirrors setup_engine: a y/z plane that
// does not fit one CTA is costed as the split path's plane buffer, which is
// larger than the cluster path's slots.
int dda_footprint(const dda_problem* p, int precision, int64_t* resident, int64_t* peak) {
  if (!p || precision < DDA_PREC_FP64 || precision > DDA_PREC_MIXED || p->max_rhs < 1) return DDA_ERR_ARG;
  const long long Gx = p->grid[0], Gy = p->grid[1], Gz = p->grid[2];
  const long long bx = p->box[0], by = p->box[1], bz = p->box[2];
  (void)bx;
  const long long nv = p->nv, nvs = (nv + 15) / 16 * 16, nl = by * bz, R = p->max_rhs;
  const long long nmat = std::max<uint32_t>(1, p->nmat);
  const bool planned = has_tuned_plan((int)Gx) && has_tuned_plan((int)Gy) && has_tuned_plan((int)Gz) &&
                       !(p->flags & DDA_FLAG_RUNTIME_PLANS);
  long long bytes = 4 * (nl + 1) + 9 * nv;                    // line offsets, dipoles, permutation, materials
  bytes += 6 * (Gx + Gy + Gz) * (8 + 16 + 4 + 4);              // plans
  auto engine = [&](long long s) {
    long long e = (Gx / 2 + 1) * (Gy / 2 + 1) * (Gz / 2 + 1) * 6 * s;  // D-hat octant
    // vectors: 10 Krylov + io; MIXED keeps two more in FP64 (x, b) and only
    // the matvec input and io in FP32
    const long long nvec = precision != DDA_PREC_MIXED ? 11 : s == 16 ? 13 : 2;
    e += R * nmat * 3 * s + R * Gx * 3 * nl * s + nvec * R * 3 * nvs * s;
    const long long q = 3 * by + ((3 * by) % 2 == 0 ? 1 : 0);
    const long long smem_yz = (Gz + Gy + Gz * q + 3 * (Gy + 1)) * s;
    bool fused_len = false;
#define C(N) fused_len = fused_len || Gy == N;
    DDA_FUSED_LENGTHS(C)
#undef C
    const bool has_yz = !planned || (Gy == Gz && fused_len);
    if (!(has_yz && smem_yz <= (long long)kSmemMax) || (p->flags & (DDA_FLAG_SPLIT_YZ | DDA_FLAG_SLOT_YZ)))
      e += R * Gx * 3 * Gz * by * s;
    return e;
  };
  if (precision != DDA_PREC_FP32) bytes += engine(16);
  if (precision != DDA_PREC_FP64) bytes += engine(8);
  // the x tiles are at least half their 72 KB maximum (pick_x_tile)
  const long long sx = precision == DDA_PREC_FP32 ? 8 : 16;
  const long long tl = std::max(1, x_tile_max(sx, Gx) / 2);
  const long long tiles = (nl + tl - 1) / tl;
  bytes += R * std::max(3 * tiles, (long long)kVecPartsMax) * (long long)sizeof(RedSums) + R * 4;
  bytes += 2 * R * (long long)sizeof(KrylovState) + R * 100000LL * 8;
  if (resident) *resident = bytes;
  const long long tmp = p->dmatrix ? (Gx / 2 + 1) * (Gy / 2 + 1) * (Gz / 2 + 1) * 6 * 16 : Gx * Gy * Gz * 16;
  if (peak) *peak = bytes + tmp;
  return DDA_OK;
}

int dda_matvec_layout(const dda_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return DDA_ERR_ARG;
  auto fill = [&](const auto& e) {
    out[0] = e.fused ? 0 : e.slot_path ? 1 : 2;
    out[1] = e.fused ? (e.yz_pair ? 2 : 1) : e.ncl;
    out[2] = e.fused ? e.yz_groups : e.cl;
    out[3] = e.slot_path ? e.sg.nrw : e.yz.nrw;
    out[4] = (int64_t)(e.fused ? e.smem_yz : e.slot_path ? e.smem_slot : e.smem_rows);
  };
  if (ctx->e32.on) fill(ctx->e32);
  else fill(ctx->e64);
  out[5] = ctx->e32.on ? ctx->e32.tl : ctx->e64.tl;
  out[6] = ctx->planned ? 1 : 0;
  out[7] = (int64_t)ctx->dev_bytes;
  return DDA_OK;
}

int dda_profile_matvec(dda_ctx* ctx, int nrhs, int reps, double* ms) {
  if (!ctx || !ms || reps < 1) return DDA_ERR_ARG;
  return guard(ctx, [&]() -> int {
    if (nrhs < 1 || nrhs > ctx->max_rhs) throw DdaError(DDA_ERR_ARG, "bad nrhs");
    if (ctx->e32.on) profile_t<float>(ctx, nrhs, reps, ms);
    else profile_t<double>(ctx, nrhs, reps, ms);
    return DDA_OK;
  });
}

}  // extern "C"

namespace {
template <typename T>
void far_field_t(dda_ctx* c, int nrhs, const double* pol, long long ndir, const double* dirs, double* out) {
  typedef typename C2<T>::t T2;
  Engine<T>& e = eng<T>(c);
  const size_t n = (size_t)nrhs * 3 * c->g.nvs;
  if (pol) host_to_engine<T>(c, pol, e.io, n);
  double* ddirs = nullptr;
  double2* dout = nullptr;
  CK(cudaMallocAsync(&ddirs, ndir * 3 * sizeof(double), c->stream));
  CK(cudaMallocAsync(&dout, (size_t)ndir * nrhs * 3 * sizeof(double2), c->stream));
  CK(cudaMemcpyAsync(ddirs, dirs, ndir * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FfGeom g;
  g.nv = c->g.nv;
  g.nvs = c->g.nvs;
  g.by = c->g.by;
  g.nlines = c->g.nlines;
  g.bx = c->g.bx;
  g.kd = c->kd;
  g.k = c->kd / c->grid_unit;
  // DipoleGeometry::moveToCenter (DDA/DipoleGeometry.cpp:75-80)
  g.ox = -((double)c->g.bx - 1) / 2 * c->grid_unit;
  g.oy = -((double)c->g.by - 1) / 2 * c->grid_unit;
  g.oz = -((double)c->g.bz - 1) / 2 * c->grid_unit;
  constexpr int DB = 4, NT = 256;
  const size_t smem = (size_t)DB * g.bx * sizeof(double2);
  if (smem > kSmemMax) throw DdaError(DDA_ERR_UNSUPPORTED, "box too long for the far-field tables");
  CK(allow_smem((const void*)k_farfield<T, NT, DB>));
  k_farfield<T, NT, DB><<<dim3((unsigned)((ndir + DB - 1) / DB), nrhs), NT, smem, c->stream>>>(
      e.io, c->line_off, c->dip, c->perm, ddirs, (int)ndir, g, dout);
  CK(cudaGetLastError());
  c->launches++;
  CK(cudaMemcpyAsync(out, dout, (size_t)ndir * nrhs * 3 * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(ddirs, c->stream));
  CK(cudaFreeAsync(dout, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

// Far field without any allocation (dda_far_field_noalloc).  The device
// copies of the directions and of the fields live in one file-scope device
// array that is part of the module image, so it exists once the module is
// loaded and no call allocates it.  Layout: directions at offset 0
// (24*ndir bytes, rounded up to 256), fields after them (48*ndir*nrhs
// bytes).  Nothing in it needs to start at zero: each call writes every
// byte it later reads.  One array per device, shared by every context on
// that device, so calls that overlap in time race on it.
constexpr size_t kFfScratchBytes = size_t(1) << 20;
static __device__ __align__(256) unsigned char g_ff_scratch[kFfScratchBytes];

constexpr int kFfMaxDevices = 64;
std::mutex g_ff_scratch_mu;
unsigned char* g_ff_scratch_ptr[kFfMaxDevices];

size_t ff_noalloc_bytes(long long ndir, int nrhs) {
  return (((size_t)ndir * 3 * sizeof(double) + 255) & ~(size_t)255) + (size_t)ndir * nrhs * 3 * sizeof(double2);
}

// Address of the scratch on `device`, which must be the current device.
// Looked up once per device, on the first call there.
unsigned char* ff_scratch(int device) {
  if (device < 0 || device >= kFfMaxDevices)
    throw DdaError(DDA_ERR_UNSUPPORTED, "device ordinal beyond the no-allocation far-field table");
  std::lock_guard<std::mutex> lock(g_ff_scratch_mu);
  if (!g_ff_scratch_ptr[device]) {
    void* ptr = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress((void**)&ptr, g_ff_scratch);
    if (rc != cudaSuccess || !ptr)
      throw DdaError(DDA_ERR_CUDA, std::string("cudaGetSymbolAddress of the far-field scratch: ") +
                                       cudaGetErrorString(rc));
    g_ff_scratch_ptr[device] = static_cast<unsigned char*>(ptr);
  }
  return g_ff_scratch_ptr[device];
}

template <typename T>
void far_field_noalloc_t(dda_ctx* c, int nrhs, long long ndir, const double* dirs, double* out) {
  Engine<T>& e = eng<T>(c);
  unsigned char* scratch = ff_scratch(c->device);
  double* ddirs = reinterpret_cast<double*>(scratch);
  double2* dout = reinterpret_cast<double2*>(scratch + ((ndir * 3 * sizeof(double) + 255) & ~(size_t)255));
  CK(cudaMemcpyAsync(ddirs, dirs, ndir * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  FfGeom g;
  g.nv = c->g.nv;
  g.nvs = c->g.nvs;
  g.by = c->g.by;
  g.nlines = c->g.nlines;
  g.bx = c->g.bx;
  g.kd = c->kd;
  g.k = c->kd / c->grid_unit;
  // DipoleGeometry::moveToCenter (DDA/DipoleGeometry.cpp:75-80)
  g.ox = -((double)c->g.bx - 1) / 2 * c->grid_unit;
  g.oy = -((double)c->g.by - 1) / 2 * c->grid_unit;
  g.oz = -((double)c->g.bz - 1) / 2 * c->grid_unit;
  constexpr int DB = 4, NT = 256;
  const size_t smem = (size_t)DB * g.bx * sizeof(double2);
  if (smem > kSmemMax) throw DdaError(DDA_ERR_UNSUPPORTED, "box too long for the far-field tables");
  CK(allow_smem((const void*)k_farfield<T, NT, DB>));
  k_farfield<T, NT, DB><<<dim3((unsigned)((ndir + DB - 1) / DB), nrhs), NT, smem, c->stream>>>(
      e.io, c->line_off, c->dip, c->perm, ddirs, (int)ndir, g, dout);
  CK(cudaGetLastError());
  c->launches++;
  CK(cudaMemcpyAsync(out, dout, (size_t)ndir * nrhs * 3 * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}
}  // namespace

extern "C" {

int dda_far_field(dda_ctx* ctx, int nrhs, const double* pol, int64_t ndir, const double* dirs, double* out) {
  if (!ctx) return DDA_ERR_ARG;
  NvtxRange range("dda far field");
  return guard(ctx, [&]() -> int {
    if (nrhs < 1 || nrhs > ctx->max_rhs || ndir < 1 || !dirs || !out) throw DdaError(DDA_ERR_ARG, "bad far-field arguments");
    if (ndir > (1LL << 31) / 4) throw DdaError(DDA_ERR_ARG, "too many directions");
    if (ctx->precision == DDA_PREC_FP32) far_field_t<float>(ctx, nrhs, pol, ndir, dirs, out);
    else far_field_t<double>(ctx, nrhs, pol, ndir, dirs, out);
    return DDA_OK;
  });
}

int dda_far_field_noalloc(dda_ctx* ctx, int nrhs, int64_t ndir, const double* dirs, double* out) {
  if (!ctx) return DDA_ERR_ARG;
  return guard(ctx, [&]() -> int {
    if (nrhs < 1 || nrhs > ctx->max_rhs || ndir < 1 || !dirs || !out) throw DdaError(DDA_ERR_ARG, "bad far-field arguments");
    if (ndir > (long long)(kFfScratchBytes / 72) || ff_noalloc_bytes(ndir, nrhs) > kFfScratchBytes)
      throw DdaError(DDA_ERR_ARG, "dda_far_field_noalloc: " + std::to_string(ndir) + " directions x " +
                                      std::to_string(nrhs) + " right-hand sides exceed its fixed scratch of " +
                                      std::to_string(kFfScratchBytes) +
                                      " bytes (24 bytes per direction, rounded up to 256, + 48 per direction and right-hand side)");
    if (ctx->precision == DDA_PREC_FP32) far_field_noalloc_t<float>(ctx, nrhs, ndir, dirs, out);
    else far_field_noalloc_t<double>(ctx, nrhs, ndir, dirs, out);
    return DDA_OK;
  });
}

int dda_get_dmatrix(dda_ctx* ctx, double* out) {
  if (!ctx || !out) return DDA_ERR_ARG;
  return guard(ctx, [&]() -> int {
    const MvGeom& g = ctx->g;
    const int hx = g.Gx / 2 + 1, hy = g.Gy / 2 + 1, hz = g.Gz / 2 + 1;
    const size_t m = (size_t)hx * hy * hz * 6;
    std::vector<double2> h(m);
    if (ctx->e64.on) {
      CK(cudaMemcpyAsync(h.data(), ctx->e64.dc, m * sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
    } else {
      std::vector<float2> f(m);
      CK(cudaMemcpyAsync(f.data(), ctx->e32.dc, m * sizeof(float2), cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      for (size_t i = 0; i < m; i++) h[i] = make_double2(f[i].x, f[i].y);
    }
    const double sc = 1.0 / (ctx->grid_unit * ctx->grid_unit * ctx->grid_unit);
    for (int kx = 0; kx < g.Gx; kx++)
      for (int kz = 0; kz < g.Gz; kz++)
        for (int ky = 0; ky < g.Gy; ky++) {
          const bool fx = kx > g.Gx / 2, fy = ky > g.Gy / 2, fz = kz > g.Gz / 2;
          const int ax = fx ? g.Gx - kx : kx, ay = fy ? g.Gy - ky : ky, az = fz ? g.Gz - kz : kz;
          const double2* src = &h[(((size_t)ax * hz + az) * hy + ay) * 6];
          const double sign[6] = {1, fx != fy ? -1.0 : 1.0, fx != fz ? -1.0 : 1.0, 1, fy != fz ? -1.0 : 1.0, 1};
          double* dst = out + 2 * 6 * (ky + (size_t)g.Gy * (kz + (size_t)g.Gz * kx));
          for (int comp = 0; comp < 6; comp++) {
            dst[2 * comp] = src[comp].x * sign[comp] * sc;
            dst[2 * comp + 1] = src[comp].y * sign[comp] * sc;
          }
        }
    return DDA_OK;
  });
}

int dda_synchronize(dda_ctx* ctx) {
  if (!ctx) return DDA_ERR_ARG;
  return guard(ctx, [&]() -> int {
    CK(cudaStreamSynchronize(ctx->stream));
    return DDA_OK;
  });
}

}  // extern "C"
