// dda_oracle.cpp -- CPU restatement of the reference DDA hot path.
//
// TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
// dda_b200: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
// reference arm may load it.  The product never links or calls it.
//
// Parity status: UNPINNED against outputs of the reference itself.  The
// reference (steffen-kiess/dda) cannot be built in this environment (it needs
// Boost, FFTW3, HDF5 and omake, none of which are present) and its own tests
// compare against a live ADDA binary (DDA/test-adda.sh, DDA/compare-adda.sh)
// that is absent too, so no reference output exists to pin against.  The
// restatement is pinned instead by independent checks kept in tests/:
//   * the FFT against numpy.fft and a naive DFT,
//   * the FFT matvec against a brute-force O(nv^2) direct sum of the same
//     Green's tensor (pins the D-matrix sign, layout and 1/N normalisation),
//   * voxelisation counts against the reference fixture DDA/box_10_8_6.geom
//     and the dipole counts quoted for the reference's README workloads,
//   * DDA cross sections of spheres against the Mie series (EMSim/Mie.cpp).
//
// Every function cites the reference file:line it follows.  Third-party
// arithmetic: the reference computes FFTs with FFTW3 (un-vendored, README asks
// for ">= 3.2.2", no pinned version; call sites LinAlg/FFTWPlan.cpp:82,113).
// This file restates the published DFT definition FFTW implements
// (unnormalised, forward kernel exp(-2 pi i jk/n), backward exp(+2 pi i jk/n))
// with a recursive mixed-radix Cooley-Tukey decomposition.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef long double ldouble;
typedef std::complex<double> cd;
typedef std::complex<ldouble> cld;

namespace {

// Constants of DDA/FPConst.hpp:36-50 (ldr_b* from doi:10.1086/172396).
const ldouble kPi = 3.1415926535897932384626433832795028L;
const ldouble kTwoPi = 6.2831853071795864769252867665590056L;
const ldouble kFourPi = 12.5663706143591729538505735331180112L;
const double kLdrB1 = 1.8915316;
const double kLdrB2 = -0.1648469;
const double kLdrB3 = 1.7700004;

std::string g_error;

// ---------------------------------------------------------------- FFT ----
// Restatement of the DFT that FFTW computes (LinAlg/FFTWPlan.cpp:82,113):
// y_k = sum_j x_j exp(-/+ 2 pi i jk/n), unnormalised both ways, in the
// precision F of the reference's ftype (fftw_plan / fftwf_plan).
template <class F>
struct FftPlanT {
  typedef std::complex<F> C;
  size_t n;
  std::vector<int> factors;
  std::vector<C> tw;  // exp(-2 pi i k / n), k = 0..n-1, from long double

  explicit FftPlanT(size_t n_) : n(n_), tw(n_) {
    size_t m = n;
    for (int p : {4, 2, 3, 5, 7}) {
      while (m % p == 0) {
        factors.push_back(p);
        m /= p;
      }
    }
    for (size_t p = 11; m > 1; p += 2) {
      while (m % p == 0) {
        factors.push_back((int)p);
        m /= p;
      }
    }
    for (size_t k = 0; k < n; k++) {
      ldouble a = -kTwoPi * (ldouble)k / (ldouble)n;
      tw[k] = C((F)cosl(a), (F)sinl(a));
    }
  }

  // Recursive decimation in time: out[0..len) = DFT of in[0], in[s], ...
  void rec(const C* in, size_t stride, C* out, size_t len, size_t fi,
           bool inv, std::vector<C>& t) const {
    if (len == 1) {
      out[0] = in[0];
      return;
    }
    int p = factors[fi];
    size_t m = len / p;
    for (int q = 0; q < p; q++)
      rec(in + q * stride, stride * p, out + q * m, m, fi + 1, inv, t);
    size_t step = n / len;  // table index scale: w_len^j = w_n^(j*step)
    for (size_t k = 0; k < m; k++) {
      for (int q = 0; q < p; q++) {
        C w = tw[(q * k * step) % n];
        if (inv) w = std::conj(w);
        t[q] = out[q * m + k] * w;
      }
      for (int s = 0; s < p; s++) {
        C acc = 0;
        for (int q = 0; q < p; q++) {
          C w = tw[((size_t)q * s * m * step) % n];
          if (inv) w = std::conj(w);
          acc += t[q] * w;
        }
        out[k + m * s] = acc;
      }
    }
  }

  // In-place transform of `count` lines: line b starts at data + b*dist,
  // elements are `stride` apart.
  void exec(C* data, size_t count, size_t stride, size_t dist, bool inv) const {
    std::vector<C> a(n), b(n), t(16);
    if (factors.size() && *std::max_element(factors.begin(), factors.end()) > 16)
      t.resize(*std::max_element(factors.begin(), factors.end()));
    for (size_t c = 0; c < count; c++) {
      C* d = data + c * dist;
      for (size_t i = 0; i < n; i++) a[i] = d[i * stride];
      rec(a.data(), 1, b.data(), n, 0, inv, t);
      for (size_t i = 0; i < n; i++) d[i * stride] = b[i];
    }
  }
};
typedef FftPlanT<double> FftPlan;

std::mutex g_plan_mutex;

template <class F>
std::shared_ptr<FftPlanT<F>> plan(size_t n) {
  static std::map<size_t, std::shared_ptr<FftPlanT<F>>> plans;
  std::lock_guard<std::mutex> lock(g_plan_mutex);
  auto it = plans.find(n);
  if (it != plans.end()) return it->second;
  auto p = std::make_shared<FftPlanT<F>>(n);
  plans[n] = p;
  return p;
}

// ------------------------------------------------------------ fftFit ----
// DDA/DDAParams.cpp:45-90.
uint32_t fftFit(uint32_t x, uint32_t override, bool supportNonPot) {
  if (override != 0) return override;
  if (x == 0) return 0;
  if (!supportNonPot) {
    uint32_t ret = 1;
    while (x > 1) {
      ret *= 2;
      x = (x + 1) / 2;
    }
    return ret;
  }
  uint32_t ret = x;
  if (ret % 2 == 1) ret++;
  for (;;) {
    uint32_t y = ret;
    while (y % 2 == 0) y /= 2;
    while (y % 3 == 0) y /= 3;
    while (y % 5 == 0) y /= 5;
    while (y % 7 == 0) y /= 7;
    if (y == 1) return ret;
    ret += 2;
  }
}

uint32_t roundUp(uint32_t v, uint32_t d) { return ((v + d - 1) / d) * d; }

}  // namespace

// ============================================================ geometry ====
// DipoleGeometry (DDA/DipoleGeometry.hpp:49-156): positions (x,y,z) as u32,
// 0-based material index per dipole, bounding box, ldouble grid unit.
struct orc_geom {
  ldouble gridUnit = 0;
  uint32_t box[3] = {0, 0, 0};
  uint32_t matCount = 0;
  std::vector<uint32_t> pos;  // nv*3 interleaved x,y,z
  std::vector<uint8_t> mat;
  bool ok = true;

  // DDA/DipoleGeometry.cpp:90-107
  void addDipole(uint32_t x, uint32_t y, uint32_t z, uint8_t m) {
    if (!(box[2] <= z + 1)) {  // positions must be sorted by z
      ok = false;
      g_error = "dipoles not sorted by z";
    }
    pos.push_back(x);
    pos.push_back(y);
    pos.push_back(z);
    mat.push_back(m);
    if (x >= box[0]) box[0] = x + 1;
    if (y >= box[1]) box[1] = y + 1;
    if (z >= box[2]) box[2] = z + 1;
    if (m >= matCount) matCount = m + 1u;
  }
};

extern "C" {

const char* orc_last_error() { return g_error.c_str(); }

// EMSim/Length.cpp:30-67: a number parsed as long double, times a unit
// factor in long double.  Returns 0 on success.
int orc_parse_number(const char* s, ldouble* out) {
  std::istringstream in(s);
  ldouble value;
  in >> value;
  if (in.fail()) return -1;
  *out = value;
  return 0;
}

int orc_parse_length(const char* s, ldouble* out) {
  std::istringstream in(s);
  ldouble value;
  in >> value;
  if (in.fail()) return -1;
  std::string unit;
  std::getline(in, unit);
  ldouble factor;
  if (unit.empty() && value == 0) {
    *out = 0;
    return 0;
  } else if (unit == "um" || unit == "\xc2\xb5m") {
    factor = 1e-6L;
  } else if (unit == "nm") {
    factor = 1e-9L;
  } else if (unit == "mm") {
    factor = 1e-3L;
  } else if (unit == "m") {
    factor = 1e+0L;
  } else {
    return -1;
  }
  *out = value * factor;
  return 0;
}

// Unnormalised in-place DFT of `count` contiguous lines of length n
// (complex interleaved), the transform the reference gets from FFTW.
void orc_fft(double* data, uint32_t n, uint32_t count, int inverse) {
  plan<double>(n)->exec(reinterpret_cast<cd*>(data), count, 1, n, inverse != 0);
}

uint32_t orc_fft_fit(uint32_t x, uint32_t override, int supportNonPot) {
  return fftFit(x, override, supportNonPot != 0);
}

// DDA/Shapes.cpp:53-73 (sphere): radius in grid units as double, dipole at
// cell centre (x - r + 0.5) kept when inside r^2; loops z, y, x.
orc_geom* orc_geom_sphere(ldouble radius, ldouble gridUnit) {
  orc_geom* g = new orc_geom;
  g->gridUnit = gridUnit;
  double r = static_cast<double>(radius / gridUnit);
  double diameter = r * 2;
  double r2 = r * r;
  for (uint32_t z = 0; z < diameter; z++)
    for (uint32_t y = 0; y < diameter; y++)
      for (uint32_t x = 0; x < diameter; x++) {
        double xd = x - r + 0.5;
        double yd = y - r + 0.5;
        double zd = z - r + 0.5;
        if (xd * xd + yd * yd + zd * zd <= r2) g->addDipole(x, y, z, 0);
      }
  return g;
}

// DDA/Shapes.cpp:91-111 (cylinder along x).
orc_geom* orc_geom_cylinder(ldouble length, ldouble radius, ldouble gridUnit) {
  orc_geom* g = new orc_geom;
  g->gridUnit = gridUnit;
  double len = static_cast<double>(length / gridUnit);
  double r = static_cast<double>(radius / gridUnit);
  double diameter = r * 2;
  double r2 = r * r;
  for (uint32_t z = 0; z < diameter; z++)
    for (uint32_t y = 0; y < diameter; y++) {
      double yd = y - r + 0.5;
      double zd = z - r + 0.5;
      if (yd * yd + zd * zd <= r2)
        for (uint32_t x = 0; x < len; x++) g->addDipole(x, y, z, 0);
    }
  return g;
}

// DDA/Shapes.cpp:130-143 (box): extent / grid unit in long double.
orc_geom* orc_geom_box(ldouble sx, ldouble sy, ldouble sz, ldouble gridUnit) {
  orc_geom* g = new orc_geom;
  g->gridUnit = gridUnit;
  ldouble s[3] = {sx / gridUnit, sy / gridUnit, sz / gridUnit};
  for (uint32_t z = 0; z < s[2]; z++)
    for (uint32_t y = 0; y < s[1]; y++)
      for (uint32_t x = 0; x < s[0]; x++) g->addDipole(x, y, z, 0);
  return g;
}

// DDA/Load.cpp:37-69: "x y z [m]" lines, '#' and 'N' lines skipped,
// materials 1-based in the file (default 1).
orc_geom* orc_geom_load_text(const char* path, ldouble gridUnit) {
  std::ifstream in(path);
  if (!in) {
    g_error = std::string("cannot open ") + path;
    return nullptr;
  }
  orc_geom* g = new orc_geom;
  g->gridUnit = gridUnit;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#' || line[0] == 'N') continue;
    std::istringstream ls(line);
    long long x, y, z, m = 1;
    if (!(ls >> x)) continue;
    if (!(ls >> y >> z)) {
      g_error = "malformed dipole line";
      delete g;
      return nullptr;
    }
    if (!(ls >> m)) m = 1;
    if (!(m > 0 && m <= 256) || x < 0 || y < 0 || z < 0) {
      g_error = "bad material index or coordinate";
      delete g;
      return nullptr;
    }
    g->addDipole((uint32_t)x, (uint32_t)y, (uint32_t)z, (uint8_t)(m - 1));
  }
  if (!g->ok) {
    delete g;
    return nullptr;
  }
  return g;
}

orc_geom* orc_geom_from_arrays(const uint32_t* pos, const uint8_t* mat,
                               uint32_t nv, ldouble gridUnit) {
  orc_geom* g = new orc_geom;
  g->gridUnit = gridUnit;
  for (uint32_t i = 0; i < nv; i++)
    g->addDipole(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], mat ? mat[i] : 0);
  if (!g->ok) {
    delete g;
    return nullptr;
  }
  return g;
}

uint32_t orc_geom_nv(const orc_geom* g) { return (uint32_t)g->mat.size(); }
void orc_geom_box_size(const orc_geom* g, uint32_t* out) {
  for (int i = 0; i < 3; i++) out[i] = g->box[i];
}
uint32_t orc_geom_matcount(const orc_geom* g) { return g->matCount; }
void orc_geom_positions(const orc_geom* g, uint32_t* out) {
  std::copy(g->pos.begin(), g->pos.end(), out);
}
void orc_geom_materials(const orc_geom* g, uint8_t* out) {
  std::copy(g->mat.begin(), g->mat.end(), out);
}
void orc_geom_free(orc_geom* g) { delete g; }

}  // extern "C"

// ============================================================ problem =====
// DDAParams (DDA/DDAParams.cpp:93-214) + CoupleConstants
// (DDA/DDAParams.cpp:315-331) + D matrix + matvec + solvers, all in double.
struct orc_problem {
  // geometry
  uint32_t nv = 0, nvs = 0, box[3] = {0, 0, 0}, grid[3] = {0, 0, 0};
  std::vector<uint32_t> pos;
  std::vector<uint8_t> mat;
  uint32_t nmat = 0;
  std::vector<cld> materials;  // nmat*3 refractive index (DiagMatrix3)
  ldouble gridUnitL = 0;
  double gridUnit = 0, gridUnitVol = 0, lambda = 0, waveNum = 0, kd = 0;
  ldouble origin[3] = {0, 0, 0};  // DDA/DipoleGeometry.cpp:75-80

  // D matrix, reference layout: [Gx][Gz][Gy][6] complex (offset
  // comp + 6*(j + Gy*(k + Gz*i)), DDA/GpuMatVecInst.cl:114)
  std::vector<cd> D;
  // couple constants per material: cc, cc_sqrt, chi_inv (3 each)
  std::vector<cd> cc, ccSqrt, chiInv;

  // matvec scratch (DDA/MatVecCpu.cpp:48-50)
  std::vector<cd> X;  // Xmatrix [3][bz][by][Gx] (x fastest)

  // the --ftype float path: D computed in float (DMatrixCpu<float>), its
  // x-grid scratch, and sqrt(cc) rounded to float
  std::vector<std::complex<float>> D32, X32;

  size_t vecSize() const { return 3 * (size_t)nvs; }
  size_t N() const { return (size_t)grid[0] * grid[1] * grid[2]; }
};

namespace {

// DDA/DMatrixCpu.cpp:49-63, in the precision F of the reference's ftype.
template <class F>
std::complex<F> singleInteractionTerm(const orc_problem& p, F rx, F ry, F rz, int mu, int nu) {
  typedef std::complex<F> C;
  F rr = std::sqrt(rx * rx + ry * ry + rz * rz);
  F q[3] = {rx / rr, ry / rr, rz / rr};
  F kr = (F)p.waveNum * rr;
  F kr2 = kr * kr;
  F qmunu = q[mu] * q[nu];
  C expval = std::exp(C(0, kr)) / C(std::pow(rr, F(3)));
  C br = C(F(3) - kr2, F(-3) * kr) * qmunu;
  if (mu == nu) br += C(kr2 - F(1), kr);
  return expval * br;
}

// DDA/DMatrixCpu.cpp:65-74 (periodicity dimension 0).
template <class F>
std::complex<F> interactionTerm(const orc_problem& p, int i, int j, int k, int mu, int nu) {
  if (!i && !j && !k) return std::complex<F>(0);
  const F d = (F)p.gridUnit;
  return singleInteractionTerm<F>(p, (F)i * d, (F)j * d, (F)k * d, mu, nu);
}

uint32_t clip(int32_t n, uint32_t M) {  // DDA/DMatrixCpu.cpp:124-131
  if (n < 0) return n + M;
  if ((uint32_t)n >= M) return n - M;
  return n;
}

template <class C> inline C maybeConj(C f, bool c) { return c ? std::conj(f) : f; }

}  // namespace

extern "C" {

// DDAParams ctor (DDA/DDAParams.cpp:93-214), single process.
// materials: nmat*3 complex refractive indices as (re, im) long double pairs.
// grid_override: three values, 0 = automatic (fftFit).
orc_problem* orc_problem_create(const orc_geom* g, const ldouble* materials,
                                uint32_t nmat, ldouble lambda,
                                const uint32_t* grid_override, int supportNonPot) {
  if (!g || g->mat.empty()) {
    g_error = "empty geometry";
    return nullptr;
  }
  if (nmat < g->matCount) {
    g_error = "fewer materials than material indices";
    return nullptr;
  }
  orc_problem* p = new orc_problem;
  p->nv = (uint32_t)g->mat.size();
  p->nvs = roundUp(p->nv, 16);
  for (int i = 0; i < 3; i++) {
    p->box[i] = g->box[i];
    p->grid[i] = fftFit(g->box[i] * 2, grid_override ? grid_override[i] : 0,
                        supportNonPot != 0);
    if (p->grid[i] % 2 != 0 || p->grid[i] < 2 * p->box[i]) {
      g_error = "bad FFT grid";
      delete p;
      return nullptr;
    }
    // DipoleGeometry::moveToCenter, DDA/DipoleGeometry.cpp:75-80
    p->origin[i] = -((ldouble)(g->box[i]) - 1.0L) / 2 * g->gridUnit;
  }
  p->pos = g->pos;
  p->mat = g->mat;
  p->nmat = nmat;
  p->materials.resize(nmat * 3);
  for (uint32_t i = 0; i < nmat * 3; i++)
    p->materials[i] = cld(materials[2 * i], materials[2 * i + 1]);
  p->gridUnitL = g->gridUnit;
  p->gridUnit = (double)g->gridUnit;
  p->gridUnitVol = (double)(g->gridUnit * g->gridUnit * g->gridUnit);
  p->lambda = (double)lambda;
  p->waveNum = (double)kTwoPi / p->lambda;  // DDA/DDAParams.cpp:212-213
  p->kd = p->waveNum * p->gridUnit;
  return p;
}

void orc_problem_free(orc_problem* p) { delete p; }

void orc_problem_info(const orc_problem* p, uint32_t* out /*9*/, double* dout /*4*/) {
  out[0] = p->nv;
  out[1] = p->nvs;
  for (int i = 0; i < 3; i++) {
    out[2 + i] = p->box[i];
    out[5 + i] = p->grid[i];
  }
  out[8] = p->nmat;
  dout[0] = p->gridUnit;
  dout[1] = p->waveNum;
  dout[2] = p->kd;
  dout[3] = p->gridUnitVol;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Beam polarisation convention of DDA/Beam.cpp:33-51 (ADDA's): pol 1 is the
// "y polarisation" incPolY, pol 2 the "x polarisation" incPolX.
void orc_beam_pol(const double* propIn, int pol, double* out3, double* prop3) {
  ldouble pr[3] = {propIn[0], propIn[1], propIn[2]};
  ldouble nrm = sqrtl(pr[0] * pr[0] + pr[1] * pr[1] + pr[2] * pr[2]);
  for (int i = 0; i < 3; i++) pr[i] /= nrm;
  ldouble px[3], py[3];
  if (fabsl(pr[2]) >= (1 - 1e-6)) {
    px[0] = pr[2]; px[1] = 0; px[2] = 0;
    py[0] = 0; py[1] = 1; py[2] = 0;
  } else {
    ldouble t = sqrtl(1 - pr[2] * pr[2]);
    px[0] = pr[0] * pr[2] / t; px[1] = pr[1] * pr[2] / t; px[2] = -t;
    py[0] = -pr[1] / t; py[1] = pr[0] / t; py[2] = 0;
  }
  for (int i = 0; i < 3; i++) {
    out3[i] = (double)(pol == 1 ? py[i] : px[i]);
    if (prop3) prop3[i] = (double)pr[i];
  }
}

// CoupleConstants (DDA/DDAParams.cpp:315-331) with the CM / LDR
// polarisability of DDA/PolarizabilityDescription.cpp:65-110.
// kind: 0 = cm, 1 = ldr, 2 = ldr-avgpol.  pol: 1 or 2.
void orc_set_cc_frame(orc_problem* p, int kind, const double* prop, const double* incPol);

void orc_set_cc(orc_problem* p, int kind, const double* propIn, int pol) {
  double incPol[3], prop[3];
  orc_beam_pol(propIn, pol, incPol, prop);
  orc_set_cc_frame(p, kind, prop, incPol);
}

// The same for a propagation direction and polarisation vector already in
// the particle frame (PolarizabilityDescription.cpp:96-98, where both are
// rotated by the inverse orientation).
void orc_set_cc_frame(orc_problem* p, int kind, const double* prop, const double* incPol) {
  p->cc.assign(p->nmat * 3, 0);
  p->ccSqrt.assign(p->nmat * 3, 0);
  p->chiInv.assign(p->nmat * 3, 0);
  double temp = p->gridUnitVol / (double)kFourPi;
  for (uint32_t i = 0; i < p->nmat; i++) {
    for (int j = 0; j < 3; j++) {
      cd m = cd((double)p->materials[i * 3 + j].real(), (double)p->materials[i * 3 + j].imag());
      cd m2 = m * m;
      cd uncorrected = 3.0 * temp * (m2 - cd(1)) / (m2 + cd(2));
      cd c = uncorrected;
      if (kind != 0) {
        cd t1 = cd(0, 2.0 / 3 * p->kd * p->kd * p->kd);
        double prop2[3] = {prop[0] * prop[0], prop[1] * prop[1], prop[2] * prop[2]};
        double inc2[3] = {incPol[0] * incPol[0], incPol[1] * incPol[1], incPol[2] * incPol[2]};
        double S;
        if (kind == 2)
          S = 0.5f * (1 - (prop2[0] * prop2[0] + prop2[1] * prop2[1] + prop2[2] * prop2[2]));
        else
          S = prop2[0] * inc2[0] + prop2[1] * inc2[1] + prop2[2] * inc2[2];
        t1 += (kLdrB1 + (kLdrB2 + kLdrB3 * S) * m2) * p->kd * p->kd;
        c = uncorrected / (cd(1) - (uncorrected / p->gridUnitVol) * t1);
      }
      p->cc[i * 3 + j] = c;
      p->ccSqrt[i * 3 + j] = std::sqrt(c);
      p->chiInv[i * 3 + j] = 1.0 / (temp * (m2 - cd(1)));
    }
  }
}

void orc_get_cc(const orc_problem* p, double* cc, double* ccSqrt, double* chiInv) {
  for (size_t i = 0; i < p->cc.size(); i++) {
    if (cc) { cc[2 * i] = p->cc[i].real(); cc[2 * i + 1] = p->cc[i].imag(); }
    if (ccSqrt) { ccSqrt[2 * i] = p->ccSqrt[i].real(); ccSqrt[2 * i + 1] = p->ccSqrt[i].imag(); }
    if (chiInv) { chiInv[2 * i] = p->chiInv[i].real(); chiInv[2 * i + 1] = p->chiInv[i].imag(); }
  }
}

// Overrides the couple-constant square roots (nmat*3 complex) directly.
void orc_set_cc_sqrt(orc_problem* p, const double* ccSqrt) {
  p->ccSqrt.resize(p->nmat * 3);
  for (size_t i = 0; i < p->ccSqrt.size(); i++) p->ccSqrt[i] = cd(ccSqrt[2 * i], ccSqrt[2 * i + 1]);
}

}  // extern "C"

namespace {

// DMatrixCpu::createDMatrix, DDA/DMatrixCpu.cpp:133-205 (non-periodic), in
// the precision F of the reference's ftype.
template <class F>
void build_dmatrix_t(orc_problem* p, std::vector<std::complex<F>>& D) {
  typedef std::complex<F> C;
  const uint32_t Gx = p->grid[0], Gy = p->grid[1], Gz = p->grid[2];
  const int bx = p->box[0], by = p->box[1], bz = p->box[2];
  const size_t N = p->N();
  D.assign(6 * N, 0);
  std::vector<C> d2(N);  // [Gz][Gy][Gx], x fastest (Fortran [Gx][Gy][Gz])
  auto px = plan<F>(Gx), py = plan<F>(Gy), pz = plan<F>(Gz);
  const F scale = -(F)(Gx * (size_t)Gy * Gz);
  for (int component = 0; component < 6; component++) {
    static const int MU[6] = {0, 0, 0, 1, 1, 2}, NU[6] = {0, 1, 2, 1, 2, 2};
    int mu = MU[component], nu = NU[component];
    std::fill(d2.begin(), d2.end(), C(0));
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < (int)Gz; k++) {
      int kcor = k > (int)Gz / 2 ? k - (int)Gz : k;
      for (int j = 1 - by; j < by; j++)
        for (int i = 1 - bx; i < bx; i++)
          d2[clip(i, Gx) + Gx * (clip(j, Gy) + (size_t)Gy * k)] = interactionTerm<F>(*p, i, j, kcor, mu, nu);
    }
    // FFT along x over all Gy*Gz lines
#pragma omp parallel for schedule(dynamic)
    for (long long l = 0; l < (long long)Gy * Gz; l++) px->exec(d2.data() + l * Gx, 1, 1, Gx, false);
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < (int)Gx; i++) {
      std::vector<C> slice((size_t)Gz * Gy, 0);   // [Gy][Gz], z fastest
      std::vector<C> sliceTr((size_t)Gy * Gz, 0); // [Gz][Gy], y fastest
      for (int j = 1 - by; j < by; j++)
        for (int k = 1 - bz; k < bz; k++) {
          uint32_t y = clip(j, Gy), z = clip(k, Gz);
          slice[z + (size_t)Gz * y] = d2[i + Gx * (y + (size_t)Gy * z)];
        }
      pz->exec(slice.data(), Gy, 1, Gz, false);
      for (uint32_t y = 0; y < Gy; y++)
        for (uint32_t z = 0; z < Gz; z++) sliceTr[y + (size_t)Gy * z] = slice[z + (size_t)Gz * y];
      py->exec(sliceTr.data(), Gz, 1, Gy, false);
      for (uint32_t k = 0; k < Gz; k++)
        for (uint32_t j = 0; j < Gy; j++)
          D[component + 6 * (j + (size_t)Gy * (k + (size_t)Gz * i))] = sliceTr[j + (size_t)Gy * k] / scale;
    }
  }
}

}  // namespace

extern "C" {

void orc_build_dmatrix(orc_problem* p) {
  build_dmatrix_t<double>(p, p->D);
  p->D32.clear();
}

void orc_get_dmatrix(const orc_problem* p, double* out) {
  std::memcpy(out, p->D.data(), p->D.size() * sizeof(cd));
}
void orc_set_dmatrix(orc_problem* p, const double* in) {
  p->D32.clear();
  p->D.resize(6 * p->N());
  std::memcpy(static_cast<void*>(p->D.data()), in, p->D.size() * sizeof(cd));
}

}  // extern "C"

namespace {

// MatVecCpu::apply, DDA/MatVecCpu.cpp:67-150, in the precision F of the
// reference's ftype: vectors are SoA [x: nvs][y: nvs][z: nvs] complex
// (DDA/DDAParams.hpp:176-186); D, the x-grid scratch X and sqrt(cc) (cs,
// nmat*3) in F.
template <class F>
void matvec_t(orc_problem* p, const std::complex<F>* arg, std::complex<F>* res, int conj,
              const std::vector<std::complex<F>>& D, std::vector<std::complex<F>>& Xv,
              const std::vector<std::complex<F>>& cs) {
  typedef std::complex<F> C;
  const uint32_t Gx = p->grid[0], Gy = p->grid[1], Gz = p->grid[2];
  const uint32_t bx = p->box[0], by = p->box[1], bz = p->box[2];
  (void)bx;
  const size_t nvs = p->nvs;
  const size_t plane = (size_t)Gx * by * bz;
  Xv.assign(3 * plane, 0);  // Xmatrix[Gx][by][bz][3] Fortran
  C* X = Xv.data();
  for (uint32_t i = 0; i < p->nv; i++) {
    uint32_t x = p->pos[3 * i], y = p->pos[3 * i + 1], z = p->pos[3 * i + 2];
    for (int c = 0; c < 3; c++) {
      C r = cs[p->mat[i] * 3 + c] * maybeConj(arg[i + c * nvs], conj != 0);
      X[x + Gx * (y + (size_t)by * (z + (size_t)bz * c))] = r;
    }
  }
  auto px = plan<F>(Gx), py = plan<F>(Gy), pz = plan<F>(Gz);
#pragma omp parallel for schedule(static)
  for (long long l = 0; l < (long long)by * bz * 3; l++) px->exec(X + l * Gx, 1, 1, Gx, false);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < (int)Gx; i++) {
    std::vector<C> slices((size_t)Gz * Gy * 3, 0);   // [3][Gy][Gz] z fastest
    std::vector<C> slicesTr((size_t)Gy * Gz * 3, 0); // [3][Gz][Gy] y fastest
    for (uint32_t j = 0; j < by; j++)
      for (uint32_t k = 0; k < bz; k++)
        for (int c = 0; c < 3; c++)
          slices[k + Gz * (j + (size_t)Gy * c)] = X[i + Gx * (j + (size_t)by * (k + (size_t)bz * c))];
    for (int c = 0; c < 3; c++) pz->exec(slices.data() + (size_t)c * Gy * Gz, by, 1, Gz, false);
    for (int c = 0; c < 3; c++)
      for (uint32_t j = 0; j < Gy; j++)
        for (uint32_t k = 0; k < Gz; k++)
          slicesTr[j + Gy * (k + (size_t)Gz * c)] = slices[k + Gz * (j + (size_t)Gy * c)];
    py->exec(slicesTr.data(), (size_t)Gz * 3, 1, Gy, false);
    for (uint32_t k = 0; k < Gz; k++)
      for (uint32_t j = 0; j < Gy; j++) {
        const C* d = &D[6 * (j + (size_t)Gy * (k + (size_t)Gz * i))];
        C xv[3], yv[3];
        for (int c = 0; c < 3; c++) xv[c] = slicesTr[j + Gy * (k + (size_t)Gz * c)];
        // SymMatrix3 * Vector3, Math/SymMatrix3.hpp:86-92
        yv[0] = d[0] * xv[0] + d[1] * xv[1] + d[2] * xv[2];
        yv[1] = d[1] * xv[0] + d[3] * xv[1] + d[4] * xv[2];
        yv[2] = d[2] * xv[0] + d[4] * xv[1] + d[5] * xv[2];
        for (int c = 0; c < 3; c++) slicesTr[j + Gy * (k + (size_t)Gz * c)] = yv[c];
      }
    py->exec(slicesTr.data(), (size_t)Gz * 3, 1, Gy, true);
    for (int c = 0; c < 3; c++)
      for (uint32_t j = 0; j < Gy; j++)
        for (uint32_t k = 0; k < Gz; k++)
          slices[k + Gz * (j + (size_t)Gy * c)] = slicesTr[j + Gy * (k + (size_t)Gz * c)];
    for (int c = 0; c < 3; c++) pz->exec(slices.data() + (size_t)c * Gy * Gz, by, 1, Gz, true);
    for (uint32_t j = 0; j < by; j++)
      for (uint32_t k = 0; k < bz; k++)
        for (int c = 0; c < 3; c++)
          X[i + Gx * (j + (size_t)by * (k + (size_t)bz * c))] = slices[k + Gz * (j + (size_t)Gy * c)];
  }
#pragma omp parallel for schedule(static)
  for (long long l = 0; l < (long long)by * bz * 3; l++) px->exec(X + l * Gx, 1, 1, Gx, true);
  for (size_t i = p->nv; i < nvs; i++)
    for (int c = 0; c < 3; c++) res[i + c * nvs] = 0;
  for (uint32_t i = 0; i < p->nv; i++) {
    uint32_t x = p->pos[3 * i], y = p->pos[3 * i + 1], z = p->pos[3 * i + 2];
    for (int c = 0; c < 3; c++) {
      C r = X[x + Gx * (y + (size_t)by * (z + (size_t)bz * c))];
      C a = maybeConj(arg[i + c * nvs], conj != 0);
      res[i + c * nvs] = maybeConj(cs[p->mat[i] * 3 + c] * r + a, conj != 0);
    }
  }
}


}  // namespace

extern "C" {

void orc_matvec(orc_problem* p, const double* argD, double* resD, int conj) {
  matvec_t<double>(p, reinterpret_cast<const cd*>(argD), reinterpret_cast<cd*>(resD), conj, p->D, p->X, p->ccSqrt);
}

// Independent check (not in the reference): the same operator as a direct
// O(nv^2) sum, y_i = x_i - sqrt(cc_i) sum_{j != i} G(r_i - r_j) sqrt(cc_j) x_j,
// with G the Green's tensor of DDA/DMatrixCpu.cpp:49-63.  Pins the sign and
// the 1/N normalisation folded into D (DDA/DMatrixCpu.cpp:200).
void orc_direct_matvec(const orc_problem* p, const double* argD, double* resD) {
  const cd* arg = reinterpret_cast<const cd*>(argD);
  cd* res = reinterpret_cast<cd*>(resD);
  const size_t nvs = p->nvs;
#pragma omp parallel for schedule(dynamic)
  for (long long ii = 0; ii < (long long)p->nv; ii++) {
    size_t i = (size_t)ii;
    cd acc[3] = {0, 0, 0};
    for (size_t j = 0; j < p->nv; j++) {
      if (i == j) continue;
      int di = (int)p->pos[3 * i] - (int)p->pos[3 * j];
      int dj = (int)p->pos[3 * i + 1] - (int)p->pos[3 * j + 1];
      int dk = (int)p->pos[3 * i + 2] - (int)p->pos[3 * j + 2];
      cd xj[3];
      for (int c = 0; c < 3; c++) xj[c] = p->ccSqrt[p->mat[j] * 3 + c] * arg[j + c * nvs];
      for (int mu = 0; mu < 3; mu++)
        for (int nu = 0; nu < 3; nu++)
          acc[mu] += interactionTerm<double>(*p, di, dj, dk, std::min(mu, nu), std::max(mu, nu)) * xj[nu];
    }
    for (int c = 0; c < 3; c++)
      res[i + c * nvs] = arg[i + c * nvs] - p->ccSqrt[p->mat[i] * 3 + c] * acc[c];
  }
  for (size_t i = p->nv; i < nvs; i++)
    for (int c = 0; c < 3; c++) res[i + c * nvs] = 0;
}

// PlaneWave::createEInc, DDA/Beam.cpp:111-118: E = exp(i k r.prop) * pol
// with r the dipole coordinate in the particle frame
// (DDA/DipoleGeometry.hpp:105-109).
void orc_einc(const orc_problem* p, const double* propIn, int pol, double* outD) {
  cd* out = reinterpret_cast<cd*>(outD);
  double incPol[3], prop[3];
  orc_beam_pol(propIn, pol, incPol, prop);
  std::fill(out, out + p->vecSize(), cd(0));
  for (uint32_t i = 0; i < p->nv; i++) {
    double c[3];
    for (int a = 0; a < 3; a++)
      c[a] = (double)((ldouble)(double)p->origin[a] + (ldouble)(double)p->pos[3 * i + a] * p->gridUnitL);
    double ph = p->waveNum * (c[0] * prop[0] + c[1] * prop[1] + c[2] * prop[2]);
    cd e = std::exp(cd(0, ph));
    for (int a = 0; a < 3; a++) out[i + a * p->nvs] = e * incPol[a];
  }
}

// Dipole coordinates [nv][3] in metres, origin at the box centre
// (DipoleGeometry::getDipoleCoordPartRef as the incident fields use it,
// DDA/Beam.cpp:116, 209).
void orc_coords(const orc_problem* p, double* out) {
  for (uint32_t i = 0; i < p->nv; i++)
    for (int a = 0; a < 3; a++)
      out[3 * i + a] = (double)((ldouble)(double)p->origin[a] + (ldouble)(double)p->pos[3 * i + a] * p->gridUnitL);
}

}  // extern "C"

// ============================================================ solvers =====
// The CPU solvers in the precision F of the reference's ftype: vectors,
// dot products and scalar recurrences in F (std::complex<F>), as
// QmrCs<F>, BicgStab<F>, BicgCs<F> and Cgnr<F> compute them, with the long
// double temporaries BicgStab uses.
namespace {

template <class F> using VecT = std::vector<std::complex<F>>;

template <class F>
F vnorm(const VecT<F>& v) {  // LinAlg/LinComb.hpp:67-73
  F r = 0;
  for (const std::complex<F>& x : v) r += std::norm(x);
  return r;
}
template <class F>
std::complex<F> vecProdConj(const VecT<F>& a, const VecT<F>& b) {  // DDA/QmrCs.cpp:48-55 (bilinear)
  std::complex<F> s = 0;
  for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
  return s;
}
template <class F>
std::complex<F> vecProd(const VecT<F>& a, const VecT<F>& b) {  // DDA/BicgStab.cpp:34-41 (Hermitian)
  std::complex<F> s = 0;
  for (size_t i = 0; i < a.size(); i++) s += a[i] * std::conj(b[i]);
  return s;
}

template <class F>
struct SolveCtx {
  typedef std::complex<F> C;
  typedef VecT<F> Vec;
  orc_problem* p;
  const std::vector<C>& D;
  std::vector<C>& X;
  std::vector<C> cs;  // sqrt(cc) per material and axis, in F
  Vec A, r, x, t1, t2, t3, t4;
  F residScale = 0, epsB = 0, inprodR = 0;
  std::vector<double> history;
  int status = 0;
  std::string msg;

  SolveCtx(orc_problem* p_, const std::vector<C>& D_, std::vector<C>& X_) : p(p_), D(D_), X(X_) {
    size_t n = p->vecSize();
    A.assign(n, 0); r.assign(n, 0); x.assign(n, 0);
    t1.assign(n, 0); t2.assign(n, 0); t3.assign(n, 0); t4.assign(n, 0);
    for (const cd& c : p->ccSqrt) cs.push_back(C(c));
  }
  void matvec(const Vec& a, Vec& out, bool conj) { matvec_t<F>(p, a.data(), out.data(), conj, D, X, cs); }
  // multMat / multMatInv, DDA/DDAParams.hpp:188-210
  void multCc(const Vec& in, Vec& out, bool inverse) {
    for (uint32_t i = 0; i < p->nv; i++)
      for (int c = 0; c < 3; c++) {
        C s = cs[p->mat[i] * 3 + c];
        out[i + c * p->nvs] = inverse ? in[i + c * p->nvs] / s : s * in[i + c * p->nvs];
      }
  }
  bool fail(int code, const char* m) {
    status = code;
    msg = m;
    return false;
  }
};

// CpuIterativeSolver::initGeneral, DDA/CpuIterativeSolver.cpp:45-91.
template <class F>
F initGeneral(SolveCtx<F>& s, const VecT<F>& einc, const VecT<F>& start) {
  typedef std::complex<F> C;
  VecT<F>& pvec = s.t1;
  std::fill(pvec.begin(), pvec.end(), C(0));
  s.multCc(einc, pvec, false);
  F temp = vnorm(pvec);
  s.residScale = 1 / temp;
  F inprodR;
  if (!start.empty()) {
    s.multCc(start, s.x, true);
    s.matvec(s.x, s.A, false);
    for (size_t i = 0; i < pvec.size(); i++) s.r[i] = s.A[i] * C(-1) + pvec[i];
    inprodR = vnorm(s.r);
  } else {
    s.matvec(pvec, s.A, false);
    for (size_t i = 0; i < pvec.size(); i++) s.r[i] = s.A[i] * C(-1) + pvec[i];
    inprodR = vnorm(s.r);
    if (temp < inprodR) {
      std::fill(s.x.begin(), s.x.end(), C(0));
      std::swap(s.r, pvec);
      inprodR = temp;
    } else {
      std::swap(s.x, pvec);
    }
  }
  return inprodR;
}

// ---- QMR-CS, DDA/QmrCs.cpp:58-168
template <class F>
struct Qmr {
  typedef std::complex<F> C;
  F omega_old, omega_new, c_old, c_new;
  C beta, mBeta, tautilda, s_old, s_new;
  void init(SolveCtx<F>& s) {
    VecT<F>& v = s.t1;
    C rvec2 = vecProdConj(s.r, s.r);
    omega_old = 0;
    beta = std::sqrt(rvec2);
    mBeta = -beta;
    omega_new = std::sqrt(s.inprodR) / std::abs(beta);
    tautilda = omega_new * beta;
    c_old = 1; c_new = 1; s_old = 0; s_new = 0;
    C bi = F(1) / beta;
    for (size_t i = 0; i < v.size(); i++) v[i] = s.r[i] * bi;
  }
  bool iteration(SolveCtx<F>& s, size_t nr, F& out) {
    VecT<F> &r = s.r, &A = s.A, &x = s.x, &v = s.t1, &vt = s.t2, &p_old = s.t3, &p_new = s.t4;
    F rtmp1 = std::norm(beta) * s.residScale;
    if (nr == 0) {
      if (rtmp1 > 1e+38f) return s.fail(-5, "QMR breakdown: beta too large");
    } else if (rtmp1 < 1e-10f || rtmp1 > 1e+38f) {
      return s.fail(-5, "QMR breakdown: beta out of range");
    }
    s.matvec(v, A, false);
    C alpha = vecProdConj(v, A);
    if (nr == 0)
      for (size_t i = 0; i < v.size(); i++) vt[i] = v[i] * (-alpha) + A[i];
    else
      for (size_t i = 0; i < v.size(); i++) vt[i] = vt[i] * mBeta + v[i] * (-alpha) + A[i];
    C ctmp3 = vecProdConj(vt, vt);
    F rtmp2 = vnorm(vt);
    C ctmp1 = omega_old * beta;
    C ctmp2 = omega_new * alpha;
    C theta = std::conj(s_old) * ctmp1;
    C eta = c_old * c_new * ctmp1 + std::conj(s_new) * ctmp2;
    C zetatilda = c_new * ctmp2 - c_old * s_new * ctmp1;
    beta = std::sqrt(ctmp3);
    mBeta = -beta;
    omega_old = omega_new;
    omega_new = std::sqrt(rtmp2) / std::abs(beta);
    F zetaabs = std::sqrt(std::norm(zetatilda) + rtmp2);
    F rtmp3 = std::sqrt(std::norm(zetatilda));
    C zeta;
    if (rtmp3 < 1e-40f) zeta = zetaabs;
    else zeta = zetaabs / rtmp3 * zetatilda;
    c_old = c_new;
    c_new = rtmp3 / zetaabs;
    s_old = s_new;
    s_new = omega_new * (beta / zeta);
    C tau = c_new * tautilda;
    tautilda = -s_new * tautilda;
    C zetaInv = F(1) / zeta;
    C mEtaZeta = -eta / zeta;
    C mThetaZeta = -theta / zeta;
    C betaInv = F(1) / beta;
    F normSNew = std::norm(s_new);
    C cNewOmegaNewTautilda = (c_new / omega_new) * tautilda;
    if (nr == 0) {
      for (size_t i = 0; i < v.size(); i++) p_new[i] = v[i] * zetaInv;
    } else {
      if (nr == 1)
        for (size_t i = 0; i < v.size(); i++) p_old[i] = p_new[i] * mEtaZeta + v[i] * zetaInv;
      else
        for (size_t i = 0; i < v.size(); i++)
          p_old[i] = p_old[i] * mThetaZeta + p_new[i] * mEtaZeta + v[i] * zetaInv;
      std::swap(p_old, p_new);
    }
    for (size_t i = 0; i < v.size(); i++) x[i] = p_new[i] * tau + x[i];
    for (size_t i = 0; i < v.size(); i++) vt[i] = vt[i] * betaInv;
    std::swap(v, vt);
    for (size_t i = 0; i < v.size(); i++) r[i] = r[i] * C(normSNew) + v[i] * cNewOmegaNewTautilda;
    out = vnorm(r);
    return true;
  }
};

// ---- BiCGStab, DDA/BicgStab.cpp:59-112 (long double for alpha, beta, omega)
template <class F>
struct BicgStab {
  typedef std::complex<F> C;
  C beta, ro_new, ro_old, omega, alpha;
  F denumOmega;
  void init(SolveCtx<F>& s) { s.t4 = s.r; }
  bool iteration(SolveCtx<F>& s, size_t nr, F& out) {
    VecT<F> &r = s.r, &A = s.A, &x = s.x, &pv = s.t1, &v = s.t2, &sv = s.t3, &rt = s.t4;
    ro_new = vecProd(r, rt);
    F dtmp = (F)(std::abs(cld(ro_new)) / (ldouble)s.inprodR);
    if (!(dtmp >= 1e-16)) return s.fail(-5, "BiCGStab breakdown: ro_new too small");
    if (nr == 0) {
      pv = r;
    } else {
      cld ro_new_alpha = cld(ro_new) * cld(alpha);
      cld ro_old_omega = cld(ro_old) * cld(omega);
      if (!(std::abs(ro_old_omega) / std::abs(ro_new_alpha) >= 10e-10))
        return s.fail(-5, "BiCGStab breakdown: omega too small");
      beta = C(ro_new_alpha / ro_old_omega);
      C mbo = -beta * omega;
      for (size_t i = 0; i < pv.size(); i++) pv[i] = pv[i] * beta + v[i] * mbo + r[i];
    }
    s.matvec(pv, v, false);
    cld vRtilda = cld(vecProd(v, rt));
    alpha = C(cld(ro_new) / vRtilda);
    for (size_t i = 0; i < v.size(); i++) sv[i] = v[i] * (-alpha) + r[i];
    F inprodRplus1 = vnorm(sv);
    if (inprodRplus1 < s.epsB) {
      for (size_t i = 0; i < v.size(); i++) x[i] = pv[i] * alpha + x[i];
    } else {
      s.matvec(sv, A, false);
      denumOmega = vnorm(A);
      omega = C(cld(vecProd(sv, A)) / (ldouble)denumOmega);
      for (size_t i = 0; i < v.size(); i++) x[i] = pv[i] * alpha + sv[i] * omega + x[i];
      for (size_t i = 0; i < v.size(); i++) r[i] = A[i] * (-omega) + sv[i];
      inprodRplus1 = vnorm(r);
      ro_old = ro_new;
    }
    out = inprodRplus1;
    return true;
  }
};

// ---- BiCG-CS, DDA/BicgCs.cpp:56-84
template <class F>
struct BicgCs {
  typedef std::complex<F> C;
  C alpha, beta, ro_new, ro_old;
  F abs_ro_new;
  void init(SolveCtx<F>&) {}
  bool iteration(SolveCtx<F>& s, size_t nr, F& out) {
    VecT<F> &r = s.r, &A = s.A, &x = s.x, &pv = s.t1;
    ro_new = vecProdConj(r, r);
    abs_ro_new = std::abs(ro_new);
    F dtmp = abs_ro_new / s.inprodR;
    if (dtmp < 1e-10 || dtmp > 1e+10) return s.fail(-5, "BiCG-CS breakdown: rho out of range");
    if (nr == 0) {
      pv = r;
    } else {
      beta = ro_new / ro_old;
      for (size_t i = 0; i < pv.size(); i++) pv[i] = pv[i] * beta + r[i];
    }
    s.matvec(pv, A, false);
    C mu_k = vecProdConj(pv, A);
    F dtmp2 = std::abs(mu_k) / abs_ro_new;
    if (dtmp2 < 10e-10) return s.fail(-5, "BiCG-CS breakdown: mu too small");
    alpha = ro_new / mu_k;
    for (size_t i = 0; i < pv.size(); i++) x[i] = pv[i] * alpha + x[i];
    for (size_t i = 0; i < pv.size(); i++) r[i] = A[i] * (-alpha) + r[i];
    ro_old = ro_new;
    out = vnorm(r);
    return true;
  }
};

// ---- CGNR, DDA/Cgnr.cpp:39-73
template <class F>
struct Cgnr {
  typedef std::complex<F> C;
  C beta;
  F ro_new, ro_old;
  void init(SolveCtx<F>&) { ro_old = 0; }
  bool iteration(SolveCtx<F>& s, size_t nr, F& out) {
    VecT<F> &r = s.r, &A = s.A, &x = s.x, &pv = s.t1;
    if (nr == 0) {
      s.matvec(r, pv, true);
      ro_new = vnorm(pv);
    } else {
      s.matvec(r, A, true);
      ro_new = vnorm(A);
      beta = ro_new / ro_old;
      for (size_t i = 0; i < pv.size(); i++) pv[i] = pv[i] * beta + A[i];
    }
    s.matvec(pv, A, false);
    C alpha = ro_new / vnorm(A);
    for (size_t i = 0; i < pv.size(); i++) x[i] = pv[i] * alpha + x[i];
    for (size_t i = 0; i < pv.size(); i++) r[i] = A[i] * (-alpha) + r[i];
    ro_old = ro_new;
    out = vnorm(r);
    return true;
  }
};

template <class F, class S>
int runSolver(SolveCtx<F>& s, S& solver, size_t maxIter, size_t maxResIncrease,
              size_t stopAfter) {
  // IterativeSolverBase::getPolVec loop, DDA/IterativeSolverBase.cpp:53-98
  size_t count = 0, counter = 0;
  solver.init(s);
  while (s.inprodR >= s.epsB) {
    if (stopAfter && count >= stopAfter) return 1;
    if (count >= maxIter) {
      s.status = -6;
      s.msg = "Too many iterations";
      return s.status;
    } else if (counter > maxResIncrease) {
      s.status = -7;
      s.msg = "Too many iterations w/o increase";
      return s.status;
    }
    F next;
    if (!solver.iteration(s, count, next)) return s.status;
    count++;
    if (next <= s.inprodR) {
      s.inprodR = next;
      counter = 0;
    } else {
      counter++;
    }
    s.history.push_back(std::sqrt((double)s.residScale * (double)next));
  }
  return 0;
}

}  // namespace

extern "C" {

struct orc_stats {
  int64_t iterations;
  int64_t matvecs;
  double residScale;
  double inprodR;      // best |r|^2 reached
  double relResidual;  // sqrt(inprodR * residScale)
  int32_t status;
  int32_t pad;
};

}  // extern "C"

namespace {

// IterativeSolverBase::getPolVec (DDA/IterativeSolverBase.cpp:40-103)
// followed by CpuIterativeSolver::getResult (DDA/CpuIterativeSolver.cpp:93-99),
// in precision F; host vectors are FP64 complex on both sides.
template <class F>
int solve_t(orc_problem* p, const std::vector<std::complex<F>>& D, std::vector<std::complex<F>>& X, int solver,
            const double* eincD, double eps, int64_t maxIter, const double* startD, double* polOut,
            orc_stats* st, int64_t stopAfter, double* history, int64_t historyCap) {
  typedef std::complex<F> C;
  SolveCtx<F> s(p, D, X);
  size_t n = p->vecSize();
  const cd* ei = reinterpret_cast<const cd*>(eincD);
  VecT<F> einc(n), start;
  for (size_t i = 0; i < n; i++) einc[i] = C(ei[i]);
  if (startD) {
    const cd* sd = reinterpret_cast<const cd*>(startD);
    start.resize(n);
    for (size_t i = 0; i < n; i++) start[i] = C(sd[i]);
  }
  s.inprodR = initGeneral(s, einc, start);
  s.epsB = (F)(eps * eps) / s.residScale;
  int rc;
  static const size_t maxInc[4] = {50000, 30000, 50000, 10};
  if (solver < 0 || solver > 3) {
    g_error = "unknown solver";
    return -1;
  }
  size_t mi = maxIter > 0 ? (size_t)maxIter : (size_t)-1;
  if (solver == 0) { Qmr<F> q; rc = runSolver(s, q, mi, maxInc[0], stopAfter); }
  else if (solver == 1) { BicgStab<F> q; rc = runSolver(s, q, mi, maxInc[1], stopAfter); }
  else if (solver == 2) { BicgCs<F> q; rc = runSolver(s, q, mi, maxInc[2], stopAfter); }
  else { Cgnr<F> q; rc = runSolver(s, q, mi, maxInc[3], stopAfter); }
  if (rc < 0) g_error = s.msg;
  if (polOut) {
    VecT<F> pv(n, 0);
    s.multCc(s.x, pv, false);
    cd* out = reinterpret_cast<cd*>(polOut);
    for (size_t i = 0; i < n; i++) out[i] = cd(pv[i]);
  }
  if (st) {
    st->iterations = (int64_t)s.history.size();
    st->residScale = s.residScale;
    st->inprodR = s.inprodR;
    st->relResidual = std::sqrt((double)s.inprodR * (double)s.residScale);
    st->status = rc;
  }
  if (history)
    for (size_t i = 0; i < s.history.size() && (int64_t)i < historyCap; i++) history[i] = s.history[i];
  return rc;
}

}  // namespace

extern "C" {

// solver: 0 = qmr, 1 = bicgstab, 2 = bicg (BiCG-CS), 3 = cgnr.
// stop_after > 0 stops after that many iterations (a bounded timing sample;
// status 1).  history (may be NULL) receives up to history_cap RE_ values.
int orc_solve(orc_problem* p, int solver, const double* eincD, double eps,
              int64_t maxIter, const double* startD, double* polOut,
              orc_stats* st, int64_t stopAfter, double* history,
              int64_t historyCap) {
  return solve_t<double>(p, p->D, p->X, solver, eincD, eps, maxIter, startD, polOut, st, stopAfter, history,
                         historyCap);
}

// The same solve on the reference's --ftype float CPU path: D (DMatrixCpu<float>,
// built on first use), the matvec (MatVecCpu<float>) and the solver
// (QmrCs<float>, ...) in float.
int orc_solve_f32(orc_problem* p, int solver, const double* eincD, double eps,
                  int64_t maxIter, const double* startD, double* polOut,
                  orc_stats* st, int64_t stopAfter, double* history,
                  int64_t historyCap) {
  if (p->D32.empty()) build_dmatrix_t<float>(p, p->D32);
  return solve_t<float>(p, p->D32, p->X32, solver, eincD, eps, maxIter, startD, polOut, st, stopAfter, history,
                        historyCap);
}

}  // extern "C"

// ========================================================= post-process ===
extern "C" {

// CpuFieldCalculator::calcField (DDA/CpuFieldCalculator.cpp:48-98): scattered
// far field in direction n (particle frame) of polarisations pvec:
// E = i k^2 exp(-i k origin.n) (S - n (n.S)), S = sum_j P_j exp(-i kd n.r_j).
void orc_calc_field(const orc_problem* p, const double* pvecD, const double* n, double* out6) {
  const cd* pv = reinterpret_cast<const cd*>(pvecD);
  cd sum[3] = {0, 0, 0};
  for (uint32_t j = 0; j < p->nv; j++) {
    const double ph = -p->kd * (n[0] * p->pos[3 * j] + n[1] * p->pos[3 * j + 1] + n[2] * p->pos[3 * j + 2]);
    const cd a = std::polar(1.0, ph);
    for (int c = 0; c < 3; c++) sum[c] += pv[j + c * p->nvs] * a;
  }
  const cd ndots = n[0] * sum[0] + n[1] * sum[1] + n[2] * sum[2];
  double on = 0;
  for (int c = 0; c < 3; c++) on += (double)p->origin[c] * n[c];
  const cd f = cd(0, p->waveNum * p->waveNum) * std::polar(1.0, -p->waveNum * on);
  for (int c = 0; c < 3; c++) {
    const cd e = f * (sum[c] - n[c] * ndots);
    out6[2 * c] = e.real();
    out6[2 * c + 1] = e.imag();
  }
}

// PlaneWave::extCross (DDA/Beam.cpp:126-133) and AbsCross::absCross
// (DDA/AbsCross.cpp:28-48) for the couple constants currently set.
void orc_cross_sections(const orc_problem* p, const double* pvecD, const double* propIn, int pol,
                        double* cext, double* cabs) {
  double incPol[3], prop[3];
  orc_beam_pol(propIn, pol, incPol, prop);
  double e[6];
  orc_calc_field(p, pvecD, prop, e);
  double s = -(e[0] * incPol[0] + e[2] * incPol[1] + e[4] * incPol[2]);
  *cext = s * (double)kFourPi / p->waveNum;
  const cd* pv = reinterpret_cast<const cd*>(pvecD);
  const double temp1 = std::pow(p->waveNum, 3.0) * 2 / 3;
  double sum = 0;
  for (uint32_t i = 0; i < p->nv; i++)
    for (int c = 0; c < 3; c++) {
      const double mdr = -std::imag(1.0 / p->cc[p->mat[i] * 3 + c]) - temp1;
      sum += mdr * std::norm(pv[i + c * p->nvs]);
    }
  *cabs = (double)kFourPi * p->waveNum * sum;
}

// Jones far field (DDA/FarFieldCalc.cpp:119-160, EMSim/JonesCalculus.cpp:74-86)
// from the polarisations of the two incident polarisations (no symmetry
// shortcut): jones[i] = {S11, S12, S21, S22} complex for angle i.
void orc_jones(const orc_problem* p, const double* pol1, const double* pol2, const double* propIn,
               const double* theta, const double* phi, int64_t count, double* jones) {
  double px[3], py[3], prop[3];
  orc_beam_pol(propIn, 2, px, prop);  // incPolX = polarisation 2
  orc_beam_pol(propIn, 1, py, nullptr);  // incPolY = polarisation 1
#pragma omp parallel for schedule(dynamic)
  for (long long i = 0; i < count; i++) {
    const double st = std::sin(theta[i]), ct = std::cos(theta[i]);
    const double sp = std::sin(phi[i]), cp = std::cos(phi[i]);
    double n[3], perp[3], par[3];
    for (int a = 0; a < 3; a++) {
      n[a] = ct * prop[a] + st * (cp * px[a] + sp * py[a]);
      perp[a] = sp * px[a] - cp * py[a];
      par[a] = -st * prop[a] + ct * (cp * px[a] + sp * py[a]);
    }
    cd fpar[2], fperp[2];
    const double* pols[2] = {pol1, pol2};
    for (int k = 0; k < 2; k++) {
      double e[6];
      orc_calc_field(p, pols[k], n, e);
      cd ev[3] = {cd(e[0], e[1]), cd(e[2], e[3]), cd(e[4], e[5])};
      fpar[k] = ev[0] * par[0] + ev[1] * par[1] + ev[2] * par[2];
      fperp[k] = ev[0] * perp[0] + ev[1] * perp[1] + ev[2] * perp[2];
    }
    cd out[4] = {cp * fpar[1] + sp * fpar[0], sp * fpar[1] - cp * fpar[0],
                 cp * fperp[1] + sp * fperp[0], sp * fperp[1] - cp * fperp[0]};
    for (int k = 0; k < 4; k++) {
      jones[8 * i + 2 * k] = out[k].real();
      jones[8 * i + 2 * k + 1] = out[k].imag();
    }
  }
}

// Bohren & Huffman BHMIE efficiencies as restated in EMSim/Mie.cpp:41-174
// (long double): size parameter x, relative index m.
void orc_mie(double xD, double mre, double mim, double* qext, double* qsca, double* qabs) {
  typedef long double f;
  typedef std::complex<f> c;
  const f x = xD;
  const c refrel(mre, mim);
  const c cxy = x * refrel;
  const f xstop = x + 4 * std::pow(x, (f)1 / 3) + 2;
  const size_t nstop = (size_t)xstop;
  const f ymod = std::abs(cxy);
  const size_t nmx = (size_t)(std::max(xstop, ymod) + 15);
  std::vector<c> cxd(nmx);
  cxd[nmx - 1] = 0;
  for (size_t i = nmx - 1; i > 0; i--) cxd[i - 1] = f(i + 1) / cxy - c(1) / (cxd[i] + f(i + 1) / cxy);
  f psi0 = std::cos(x), psi1 = std::sin(x), chi0 = -std::sin(x), chi1 = std::cos(x);
  f apsi1 = psi1;
  c cxxi1 = c(apsi1, -chi1);
  f qs = 0;
  c s1fwd = 0;
  for (size_t n = 0; n < nstop; n++) {
    const f rn = n + 1;
    const f fn = (2 * rn + 1) / (rn * (rn + 1));
    const f psi = (2 * rn - 1) * psi1 / x - psi0;
    const f chi = (2 * rn - 1) * chi1 / x - chi0;
    const c cxxi = c(psi, -chi);
    const c an = ((cxd[n] / refrel + rn / x) * psi - apsi1) / ((cxd[n] / refrel + rn / x) * cxxi - cxxi1);
    const c bn = ((refrel * cxd[n] + rn / x) * psi - apsi1) / ((refrel * cxd[n] + rn / x) * cxxi - cxxi1);
    qs += (2 * rn + 1) * (std::norm(an) + std::norm(bn));
    // forward direction (mu = 1): pi_n = tau_n = n (n+1) / 2
    const f pin = rn * (rn + 1) / 2;
    s1fwd += fn * (an * pin + bn * pin);
    psi0 = psi1; psi1 = psi; apsi1 = psi1;
    chi0 = chi1; chi1 = chi;
    cxxi1 = c(apsi1, -chi1);
  }
  *qsca = (double)((2 / (x * x)) * qs);
  *qext = (double)((4 / (x * x)) * std::real(s1fwd));
  *qabs = *qext - *qsca;
}

}  // extern "C"
