// frontend.cpp -- host-side problem setup of libdda_b200.so
// (include/dda_frontend.h): FFT grid choice, dipole-geometry voxelisation,
// couple constants and the plane-wave incident field.  Plain C++ on the host;
// the device path starts at dda_create().

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dda_frontend.h"

namespace {

typedef long double ld;
thread_local std::string g_err;

const ld kTwoPi = 6.2831853071795864769252867665590056L;
const ld kFourPi = 12.5663706143591729538505735331180112L;
// doi:10.1086/172396 (DDA/FPConst.hpp:48-50)
const double kB1 = 1.8915316, kB2 = -0.1648469, kB3 = 1.7700004;

// EMSim::Length (EMSim/Length.cpp:30-67): decimal in long double times the
// unit factor in long double.
bool parse_length(const char* s, ld* out) {
  if (!s) return false;
  std::istringstream in(s);
  ld v;
  in >> v;
  if (in.fail()) return false;
  std::string unit;
  std::getline(in, unit);
  if (unit.empty() && v == 0) { *out = 0; return true; }
  ld f;
  if (unit == "um" || unit == "\xc2\xb5m") f = 1e-6L;
  else if (unit == "nm") f = 1e-9L;
  else if (unit == "mm") f = 1e-3L;
  else if (unit == "m") f = 1e+0L;
  else return false;
  *out = v * f;
  return true;
}

}  // namespace

struct dda_geometry {
  ld grid_unit = 0;
  uint32_t box[3] = {0, 0, 0};
  uint32_t nmat = 0;
  std::vector<uint32_t> pos;
  std::vector<uint8_t> mat;
  bool sorted = true;
  // DipoleGeometry::addDipole (DDA/DipoleGeometry.cpp:90-107)
  void add(uint32_t x, uint32_t y, uint32_t z, uint8_t m) {
    if (!(box[2] <= z + 1)) sorted = false;
    pos.insert(pos.end(), {x, y, z});
    mat.push_back(m);
    if (x >= box[0]) box[0] = x + 1;
    if (y >= box[1]) box[1] = y + 1;
    if (z >= box[2]) box[2] = z + 1;
    if (m >= nmat) nmat = m + 1u;
  }
};

extern "C" {

const char* dda_frontend_error(void) { return g_err.c_str(); }

uint32_t dda_fft_fit(uint32_t x, uint32_t override_size, int support_nonpot) {
  // DDA/DDAParams.cpp:45-90
  if (override_size) return override_size;
  if (x == 0) return 0;
  if (!support_nonpot) {
    uint32_t r = 1;
    while (x > 1) { r *= 2; x = (x + 1) / 2; }
    return r;
  }
  uint32_t r = x + (x & 1u);
  for (;; r += 2) {
    uint32_t y = r;
    for (uint32_t p : {2u, 3u, 5u, 7u})
      while (y % p == 0) y /= p;
    if (y == 1) return r;
  }
}

int dda_parse_length_m(const char* s, double* metres) {
  ld v;
  if (!parse_length(s, &v)) { g_err = std::string("bad length: ") + (s ? s : "(null)"); return -1; }
  *metres = (double)v;
  return 0;
}

// Shapes (DDA/Shapes.cpp:53-143).  Each loops z, y, x so positions come out
// sorted by z as DDAParams requires (DDA/DDAParams.cpp:193-210).
int dda_geom_sphere(const char* radius, const char* grid_unit, dda_geometry** out) {
  ld R, d;
  if (!out || !parse_length(radius, &R) || !parse_length(grid_unit, &d) || !(d > 0)) {
    g_err = "sphere: bad radius or grid unit";
    return -1;
  }
  dda_geometry* g = new dda_geometry;
  g->grid_unit = d;
  const double r = static_cast<double>(R / d);
  const double diameter = r * 2, r2 = r * r;
  for (uint32_t z = 0; z < diameter; z++)
    for (uint32_t y = 0; y < diameter; y++)
      for (uint32_t x = 0; x < diameter; x++) {
        const double xd = x - r + 0.5, yd = y - r + 0.5, zd = z - r + 0.5;
        if (xd * xd + yd * yd + zd * zd <= r2) g->add(x, y, z, 0);
      }
  if (g->mat.empty()) { delete g; g_err = "the geometry has no dipoles"; return -1; }
  *out = g;
  return 0;
}

int dda_geom_cylinder(const char* length, const char* radius, const char* grid_unit,
                      dda_geometry** out) {
  ld L, R, d;
  if (!out || !parse_length(length, &L) || !parse_length(radius, &R) || !parse_length(grid_unit, &d) ||
      !(d > 0)) {
    g_err = "cylinder: bad length, radius or grid unit";
    return -1;
  }
  dda_geometry* g = new dda_geometry;
  g->grid_unit = d;
  const double len = static_cast<double>(L / d), r = static_cast<double>(R / d);
  const double diameter = r * 2, r2 = r * r;
  for (uint32_t z = 0; z < diameter; z++)
    for (uint32_t y = 0; y < diameter; y++) {
      const double yd = y - r + 0.5, zd = z - r + 0.5;
      if (yd * yd + zd * zd <= r2)
        for (uint32_t x = 0; x < len; x++) g->add(x, y, z, 0);
    }
  if (g->mat.empty()) { delete g; g_err = "the geometry has no dipoles"; return -1; }
  *out = g;
  return 0;
}

int dda_geom_box(const char* sx, const char* sy, const char* sz, const char* grid_unit,
                 dda_geometry** out) {
  ld a, b, c, d;
  if (!out || !parse_length(sx, &a) || !parse_length(sy, &b) || !parse_length(sz, &c) ||
      !parse_length(grid_unit, &d) || !(d > 0)) {
    g_err = "box: bad size or grid unit";
    return -1;
  }
  dda_geometry* g = new dda_geometry;
  g->grid_unit = d;
  const ld s[3] = {a / d, b / d, c / d};  // compared in long double
  for (uint32_t z = 0; z < s[2]; z++)
    for (uint32_t y = 0; y < s[1]; y++)
      for (uint32_t x = 0; x < s[0]; x++) g->add(x, y, z, 0);
  if (g->mat.empty()) { delete g; g_err = "the geometry has no dipoles"; return -1; }
  *out = g;
  return 0;
}

// Text dipole list (DDA/Load.cpp:37-69): "x y z [material]" with 1-based
// materials, lines starting with '#' or 'N' skipped.
int dda_geom_load(const char* path, const char* grid_unit, dda_geometry** out) {
  ld d;
  if (!out || !path || !parse_length(grid_unit, &d) || !(d > 0)) {
    g_err = "load: bad path or grid unit";
    return -1;
  }
  std::ifstream in(path);
  if (!in) { g_err = std::string("load: cannot open ") + path; return -1; }
  dda_geometry* g = new dda_geometry;
  g->grid_unit = d;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#' || line[0] == 'N') continue;
    std::istringstream ls(line);
    long long x, y, z, m = 1;
    if (!(ls >> x)) continue;
    if (!(ls >> y >> z) || x < 0 || y < 0 || z < 0) { delete g; g_err = "load: malformed line"; return -1; }
    if (!(ls >> m)) m = 1;
    if (m < 1 || m > 256) { delete g; g_err = "load: material out of range"; return -1; }
    g->add((uint32_t)x, (uint32_t)y, (uint32_t)z, (uint8_t)(m - 1));
  }
  if (!g->sorted) { delete g; g_err = "load: dipoles must be sorted by z"; return -1; }
  if (g->mat.empty()) { delete g; g_err = "the geometry has no dipoles"; return -1; }
  *out = g;
  return 0;
}

int dda_geom_from_arrays(const uint32_t* pos, const uint8_t* mat, uint32_t nv, const char* grid_unit,
                         dda_geometry** out) {
  ld d;
  if (!out || !pos || !parse_length(grid_unit, &d) || !(d > 0)) { g_err = "bad arguments"; return -1; }
  dda_geometry* g = new dda_geometry;
  g->grid_unit = d;
  for (uint32_t i = 0; i < nv; i++) g->add(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], mat ? mat[i] : 0);
  if (!g->sorted) { delete g; g_err = "dipoles must be sorted by z"; return -1; }
  if (g->mat.empty()) { delete g; g_err = "the geometry has no dipoles"; return -1; }
  *out = g;
  return 0;
}

void dda_geom_free(dda_geometry* g) { delete g; }
uint32_t dda_geom_nv(const dda_geometry* g) { return g ? (uint32_t)g->mat.size() : 0; }
uint32_t dda_geom_nmat(const dda_geometry* g) { return g ? g->nmat : 0; }
void dda_geom_box_size(const dda_geometry* g, uint32_t* box) { for (int i = 0; i < 3; i++) box[i] = g->box[i]; }
double dda_geom_grid_unit(const dda_geometry* g) { return (double)g->grid_unit; }
const uint32_t* dda_geom_positions(const dda_geometry* g) { return g->pos.data(); }
const uint8_t* dda_geom_materials(const dda_geometry* g) { return g->mat.data(); }

// Incident polarisations of DDA/Beam.cpp:33-51 (the ADDA convention): pol 1
// is "y polarisation", pol 2 "x polarisation".  prop is normalised.
void dda_beam_pol(const double* prop_in, int pol, double* inc_pol, double* prop_out) {
  ld p[3] = {prop_in[0], prop_in[1], prop_in[2]};
  const ld n = sqrtl(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
  for (auto& v : p) v /= n;
  ld x[3], y[3];
  if (fabsl(p[2]) >= 1 - 1e-6) {
    x[0] = p[2]; x[1] = 0; x[2] = 0;
    y[0] = 0; y[1] = 1; y[2] = 0;
  } else {
    const ld t = sqrtl(1 - p[2] * p[2]);
    x[0] = p[0] * p[2] / t; x[1] = p[1] * p[2] / t; x[2] = -t;
    y[0] = -p[1] / t; y[1] = p[0] / t; y[2] = 0;
  }
  for (int i = 0; i < 3; i++) {
    inc_pol[i] = (double)(pol == 1 ? y[i] : x[i]);
    if (prop_out) prop_out[i] = (double)p[i];
  }
}

// The beam's vectors in the particle frame for a particle orientation given
// as ZYZ Euler angles in degrees (--orient): R = Rz(alpha) Ry(beta) Rz(gamma)
// as a unit quaternion q (EMSim::Rotation::fromZYZDeg, EMSim/Rotation.hpp:
// 94-102), and each lab-frame vector v mapped to R^-1 v = conj(q) v q
// (DipoleGeometry::orientationInverse, DDA/DipoleGeometry.cpp:149-152;
// Beam::propP / getIncPolP, DDA/Beam.hpp:69-81).  prop_p, pol1_p, pol2_p:
// the normalised propagation direction and the polarisation vectors of
// dda_beam_pol, rotated; center_in/center_p (may be NULL): a point.
static void quat_mul(const ld a[4], const ld b[4], ld r[4]) {
  r[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  r[1] = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  r[2] = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  r[3] = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
}

void dda_beam_frame(const double* prop_in, const double* orient_deg, double* prop_p, double* pol1_p,
                    double* pol2_p, const double* center_in, double* center_p) {
  double v[4][3];
  dda_beam_pol(prop_in, 1, v[1], v[0]);
  dda_beam_pol(prop_in, 2, v[2], nullptr);
  for (int a = 0; a < 3; a++) v[3][a] = center_in ? center_in[a] : 0.0;
  const ld pi = 3.14159265358979323846264338327950288L;
  ld q[4] = {1, 0, 0, 0};
  const int axis[3] = {3, 2, 3};  // z, y, z
  for (int k = 0; k < 3; k++) {
    const ld h = (orient_deg ? (ld)orient_deg[k] : 0.0L) / 180 * pi / 2;
    ld f[4] = {cosl(h), 0, 0, 0}, t[4];
    f[axis[k]] = sinl(h);
    quat_mul(q, f, t);
    for (int i = 0; i < 4; i++) q[i] = t[i];
  }
  const ld n = sqrtl(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  for (auto& x : q) x /= n;
  const ld qc[4] = {q[0], -q[1], -q[2], -q[3]};
  double* out[4] = {prop_p, pol1_p, pol2_p, center_p};
  for (int j = 0; j < 4; j++) {
    if (!out[j]) continue;
    const ld w[4] = {0, v[j][0], v[j][1], v[j][2]};
    ld t[4], r[4];
    quat_mul(qc, w, t);
    quat_mul(t, q, r);
    for (int a = 0; a < 3; a++) out[j][a] = (double)r[a + 1];
  }
}

// Couple constants (DDA/DDAParams.cpp:315-331) with the polarisability of
// DDA/PolarizabilityDescription.cpp:65-110.  refr: nmat*3 complex refractive
// indices; outputs nmat*3 complex each (any output may be NULL).
int dda_couple_constants(int kind, uint32_t nmat, const double* refr, double grid_unit, double wave_num,
                         const double* prop_in, int pol, double* cc, double* cc_sqrt, double* chi_inv) {
  if (!prop_in) { g_err = "bad arguments"; return -1; }
  double inc[3], prop[3];
  dda_beam_pol(prop_in, pol, inc, prop);
  return dda_couple_constants_frame(kind, nmat, refr, grid_unit, wave_num, prop, inc, cc, cc_sqrt, chi_inv);
}

// The same with the propagation direction and polarisation vector given in
// the particle frame (dda_beam_frame; PolarizabilityDescription.cpp:96-98
// rotates both by the inverse orientation).
int dda_couple_constants_frame(int kind, uint32_t nmat, const double* refr, double grid_unit, double wave_num,
                               const double* prop, const double* inc, double* cc, double* cc_sqrt, double* chi_inv) {
  if (kind < DDA_POL_CM || kind > DDA_POL_LDR_AVGPOL || !refr || !prop || !inc) { g_err = "bad arguments"; return -1; }
  typedef std::complex<double> cd;
  const ld d = grid_unit;
  const double vol = (double)(d * d * d);
  const double kd = wave_num * grid_unit;
  const double temp = vol / (double)kFourPi;
  for (uint32_t i = 0; i < nmat * 3; i++) {
    const cd m(refr[2 * i], refr[2 * i + 1]);
    const cd m2 = m * m;
    const cd unc = 3.0 * temp * (m2 - cd(1)) / (m2 + cd(2));
    cd c = unc;
    if (kind != DDA_POL_CM) {
      cd t1(0, 2.0 / 3 * kd * kd * kd);
      double S;
      const double p2[3] = {prop[0] * prop[0], prop[1] * prop[1], prop[2] * prop[2]};
      if (kind == DDA_POL_LDR_AVGPOL) {
        S = 0.5f * (1 - (p2[0] * p2[0] + p2[1] * p2[1] + p2[2] * p2[2]));
      } else {
        S = p2[0] * inc[0] * inc[0] + p2[1] * inc[1] * inc[1] + p2[2] * inc[2] * inc[2];
      }
      t1 += (kB1 + (kB2 + kB3 * S) * m2) * kd * kd;
      c = unc / (cd(1) - (unc / vol) * t1);
    }
    const cd sq = std::sqrt(c), ci = 1.0 / (temp * (m2 - cd(1)));
    if (cc) { cc[2 * i] = c.real(); cc[2 * i + 1] = c.imag(); }
    if (cc_sqrt) { cc_sqrt[2 * i] = sq.real(); cc_sqrt[2 * i + 1] = sq.imag(); }
    if (chi_inv) { chi_inv[2 * i] = ci.real(); chi_inv[2 * i + 1] = ci.imag(); }
  }
  return 0;
}

// PlaneWave::createEInc (DDA/Beam.cpp:111-118): E_i = exp(i k r_i.prop) pol,
// r_i the dipole position in the particle frame with the particle centred
// (DipoleGeometry::moveToCenter, DDA/DipoleGeometry.cpp:75-80).
int dda_einc_plane(const dda_geometry* g, double wave_num, const double* prop_in, int pol, double* einc) {
  if (!prop_in) { g_err = "bad arguments"; return -1; }
  double inc[3], prop[3];
  dda_beam_pol(prop_in, pol, inc, prop);
  return dda_einc_plane_frame(g, wave_num, prop, inc, einc);
}

// The plane wave with its propagation direction and polarisation vector in
// the particle frame (PlaneWave::createEInc with propP and getIncPolP,
// DDA/Beam.cpp:113-117).
int dda_einc_plane_frame(const dda_geometry* g, double wave_num, const double* prop, const double* inc,
                         double* einc) {
  if (!g || !prop || !inc || !einc) { g_err = "bad arguments"; return -1; }
  const uint32_t nv = (uint32_t)g->mat.size(), nvs = (nv + 15) / 16 * 16;
  std::memset(einc, 0, sizeof(double) * 2 * 3 * (size_t)nvs);
  ld origin[3];
  for (int a = 0; a < 3; a++) origin[a] = -((ld)g->box[a] - 1.0L) / 2 * g->grid_unit;
  for (uint32_t i = 0; i < nv; i++) {
    double r[3];
    for (int a = 0; a < 3; a++)
      r[a] = (double)((ld)(double)origin[a] + (ld)(double)g->pos[3 * i + a] * g->grid_unit);
    const double ph = wave_num * (r[0] * prop[0] + r[1] * prop[1] + r[2] * prop[2]);
    const double c = std::cos(ph), s = std::sin(ph);
    for (int a = 0; a < 3; a++) {
      einc[2 * (i + (size_t)a * nvs)] = c * inc[a];
      einc[2 * (i + (size_t)a * nvs) + 1] = s * inc[a];
    }
  }
  return 0;
}

// Gaussian-beam incident field (Beams::Gaussian::createEInc,
// DDA/Beam.cpp:196-263).  The beam frame: ex = the polarisation vector of
// `pol`, ey = ex rotated by +90 degrees about the propagation direction, z
// along it; coordinates relative to the beam centre, scaled by the waist w0
// across and by the confocal parameter b = k w0^2 along the beam.  With
// Q = 1 / (2 zeta - i) and psi0 = -i Q exp(i rho^2 Q), the fundamental mode
// psi0 exp(i k z) (Gouesbet, Maheu, Grehan, JOSA A 5, 1427, eq. 22) is
// corrected to third (Davis, Phys. Rev. A 19, 1177) or fifth order in
// s = 1 / (k w0) (Barton, Alexander, J. Appl. Phys. 66, 2800, eq. 25), all
// with the signs of the imaginary parts for an exp(-i omega t) time factor.
int dda_einc_gaussian(const dda_geometry* g, double wave_num, const double* prop_in, int pol, int kind,
                      double waist, const double* center, double* einc) {
  if (!prop_in || (pol != 1 && pol != 2)) {
    g_err = "bad arguments";
    return -1;
  }
  double p1[3], p2[3], prop[3];
  dda_beam_pol(prop_in, 1, p1, prop);
  dda_beam_pol(prop_in, 2, p2, nullptr);
  double ex[3], ey[3];
  for (int a = 0; a < 3; a++) {
    ex[a] = pol == 1 ? p1[a] : p2[a];
    ey[a] = pol == 1 ? -p2[a] : p1[a];
  }
  return dda_einc_gaussian_frame(g, wave_num, prop, ex, ey, kind, waist, center, einc);
}

// The Gaussian beam with its frame (prop, ex = the polarisation vector, ey)
// and centre in the particle frame (DDA/Beam.cpp:198-205 rotate all four by
// the inverse orientation).
int dda_einc_gaussian_frame(const dda_geometry* g, double wave_num, const double* prop, const double* ex,
                            const double* ey, int kind, double waist, const double* center, double* einc) {
  if (!g || !prop || !ex || !ey || !einc || !(waist > 0) || kind < DDA_BEAM_LMINUS || kind > DDA_BEAM_BARTON5) {
    g_err = "bad arguments";
    return -1;
  }
  typedef std::complex<double> cd;
  const uint32_t nv = (uint32_t)g->mat.size(), nvs = (nv + 15) / 16 * 16;
  const double c0[3] = {center ? center[0] : 0.0, center ? center[1] : 0.0, center ? center[2] : 0.0};
  const double w0 = waist, b = wave_num * w0 * w0, s = 1 / (wave_num * w0);
  const double s2 = s * s, s3 = s2 * s, s4 = s2 * s2, s5 = s4 * s;
  const cd I(0, 1);
  std::memset(einc, 0, sizeof(double) * 2 * 3 * (size_t)nvs);
  ld origin[3];
  for (int a = 0; a < 3; a++) origin[a] = -((ld)g->box[a] - 1.0L) / 2 * g->grid_unit;
  for (uint32_t i = 0; i < nv; i++) {
    double r[3];
    for (int a = 0; a < 3; a++)
      r[a] = (double)((ld)(double)origin[a] + (ld)(double)g->pos[3 * i + a] * g->grid_unit) - c0[a];
    const double x = r[0] * ex[0] + r[1] * ex[1] + r[2] * ex[2];
    const double y = r[0] * ey[0] + r[1] * ey[1] + r[2] * ey[2];
    const double z = r[0] * prop[0] + r[1] * prop[1] + r[2] * prop[2];
    const double xi = x / w0, eta = y / w0, zeta = z / b;
    const double rho2 = xi * xi + eta * eta, rho4 = rho2 * rho2;
    const cd Q = 1.0 / cd(2 * zeta, -1);
    const cd amp = -I * Q * std::exp(I * rho2 * Q) * std::exp(I * (wave_num * z));  // psi0 exp(ikz)
    cd fx = 1, fy = 0, fz = 0;
    if (kind != DDA_BEAM_LMINUS) {
      const cd Q2 = Q * Q, Q3 = Q2 * Q, Q4 = Q2 * Q2;
      const double xi2 = xi * xi;
      if (kind == DDA_BEAM_DAVIS3) {
        fx = 1.0 + s2 * (-4.0 * Q2 * xi2 - I * Q3 * rho4);
        fz = -s * 2.0 * Q * xi + s3 * (8.0 * Q3 * rho2 * xi + 2.0 * I * Q4 * rho4 * xi - 4.0 * I * Q2 * xi);
      } else {
        const cd Q5 = Q4 * Q, Q6 = Q4 * Q2, Q7 = Q6 * Q;
        fx = 1.0 + s2 * (-rho2 * Q2 - I * rho4 * Q3 - 2.0 * Q2 * xi2) +
             s4 * (2.0 * rho4 * Q4 + 3.0 * I * rho4 * rho2 * Q5 - 0.5 * rho4 * rho4 * Q6 +
                   (8.0 * rho2 * Q4 + 2.0 * I * rho4 * Q5) * xi2);
        fy = s2 * (-2.0 * Q2 * xi * eta) + s4 * ((8.0 * rho2 * Q4 + 2.0 * I * rho4 * Q5) * xi * eta);
        fz = s * (-2.0 * Q * xi) + s3 * ((6.0 * rho2 * Q3 + 2.0 * I * rho4 * Q4) * xi) +
             s5 * ((-20.0 * rho4 * Q5 - 10.0 * I * rho4 * rho2 * Q6 + rho4 * rho4 * Q7) * xi);
      }
    }
    for (int a = 0; a < 3; a++) {
      const cd e = (fx * ex[a] + fy * ey[a] + fz * prop[a]) * amp;
      einc[2 * (i + (size_t)a * nvs)] = e.real();
      einc[2 * (i + (size_t)a * nvs) + 1] = e.imag();
    }
  }
  return 0;
}

}  // extern "C"
