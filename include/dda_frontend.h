/*
 * dda_frontend.h -- host-side problem setup exported by libdda_b200.so:
 * the pieces of the reference's front end that decide what the device path
 * computes (grid size, dipole list, couple constants, incident field).
 * Return 0 on success, -1 on failure (message: dda_frontend_error()).
 */
#ifndef DDA_FRONTEND_H
#define DDA_FRONTEND_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DDA_POL_CM 0         /* Clausius-Mossotti */
#define DDA_POL_LDR 1        /* lattice dispersion relation */
#define DDA_POL_LDR_AVGPOL 2 /* LDR with avgpol */

typedef struct dda_geometry dda_geometry;

const char* dda_frontend_error(void);

/* FFT grid edge for a doubled box edge x: next even 2,3,5,7-smooth size
 * (support_nonpot != 0) or next power of two; override_size wins when
 * non-zero.  Replaces fftFit (DDA/DDAParams.cpp:45-90). */
uint32_t dda_fft_fit(uint32_t x, uint32_t override_size, int support_nonpot);

/* EMSim::Length text ("10um", "0.1um", "500nm") in metres
 * (EMSim/Length.cpp:30-67). */
int dda_parse_length_m(const char* s, double* metres);

/* Dipole geometries.  Lengths are EMSim::Length strings, evaluated in long
 * double like the reference.  Replace Shapes::Sphere / Cylinder / Box
 * ::createDipoleGeometry (DDA/Shapes.cpp:53-143), loadDipoleGeometry
 * (DDA/Load.cpp:37-69) and DipoleGeometry::addDipole
 * (DDA/DipoleGeometry.cpp:90-107). */
int dda_geom_sphere(const char* radius, const char* grid_unit, dda_geometry** out);
int dda_geom_cylinder(const char* length, const char* radius, const char* grid_unit, dda_geometry** out);
int dda_geom_box(const char* sx, const char* sy, const char* sz, const char* grid_unit, dda_geometry** out);
int dda_geom_load(const char* path, const char* grid_unit, dda_geometry** out);
int dda_geom_from_arrays(const uint32_t* positions, const uint8_t* materials, uint32_t nv,
                         const char* grid_unit, dda_geometry** out);
void dda_geom_free(dda_geometry* g);
uint32_t dda_geom_nv(const dda_geometry* g);
uint32_t dda_geom_nmat(const dda_geometry* g);
void dda_geom_box_size(const dda_geometry* g, uint32_t* box3);
double dda_geom_grid_unit(const dda_geometry* g);
const uint32_t* dda_geom_positions(const dda_geometry* g); /* nv*3, valid until free */
const uint8_t* dda_geom_materials(const dda_geometry* g);  /* nv */

/* Incident polarisation vector of polarisation 1 or 2 for a propagation
 * direction (DDA/Beam.cpp:33-51). */
void dda_beam_pol(const double* prop, int pol, double* inc_pol3, double* prop_normalised3);

/* The beam's vectors in the particle frame for the particle orientation
 * orient_deg = ZYZ Euler angles (alpha, beta, gamma) in degrees (--orient;
 * NULL: none): the normalised propagation direction prop_p and the
 * polarisation vectors of dda_beam_pol for polarisations 1 and 2, and the
 * point center_in (may be NULL) as center_p, each mapped by the inverse of
 * R = Rz(alpha) Ry(beta) Rz(gamma) (EMSim::Rotation::fromZYZDeg,
 * EMSim/Rotation.hpp:94-102; DipoleGeometry::orientationInverse,
 * DDA/DipoleGeometry.cpp:149-152).  The *_frame functions below take these. */
void dda_beam_frame(const double* prop, const double* orient_deg, double* prop_p, double* pol1_p, double* pol2_p,
                    const double* center_in, double* center_p);

/* Couple constants cc, sqrt(cc) and the inverse susceptibility for nmat*3
 * complex refractive indices (CoupleConstants, DDA/DDAParams.cpp:315-331;
 * Cm / Ldr ::getCoupleConstants, DDA/PolarizabilityDescription.cpp:65-110). */
int dda_couple_constants(int kind, uint32_t nmat, const double* refr, double grid_unit, double wave_num,
                         const double* prop, int pol, double* cc, double* cc_sqrt, double* chi_inv);
/* The same for a propagation direction and polarisation vector in the
 * particle frame (DDA/PolarizabilityDescription.cpp:96-98). */
int dda_couple_constants_frame(int kind, uint32_t nmat, const double* refr, double grid_unit, double wave_num,
                               const double* prop_p, const double* pol_p, double* cc, double* cc_sqrt,
                               double* chi_inv);

/* Plane-wave incident field [3][nvs] complex for polarisation pol
 * (PlaneWave::createEInc, DDA/Beam.cpp:111-118). */
int dda_einc_plane(const dda_geometry* g, double wave_num, const double* prop, int pol, double* einc);
/* The same for a propagation direction and polarisation vector in the
 * particle frame (DDA/Beam.cpp:113-117). */
int dda_einc_plane_frame(const dda_geometry* g, double wave_num, const double* prop_p, const double* pol_p,
                         double* einc);

#define DDA_BEAM_LMINUS 0  /* fundamental Gaussian mode */
#define DDA_BEAM_DAVIS3 1  /* Davis, third-order corrections */
#define DDA_BEAM_BARTON5 2 /* Barton-Alexander, fifth-order corrections */

/* Gaussian-beam incident field [3][nvs] complex for polarisation pol: waist
 * radius `waist` (metres), beam centre `center` (3 doubles, metres, relative
 * to the target centre; NULL: the origin), propagation direction prop
 * (Beams::Gaussian::createEInc, DDA/Beam.cpp:196-263; --beam
 * gaussian:<kind>,<waist>[,(x,y,z)], DDA/Beam.cpp:139-181). */
int dda_einc_gaussian(const dda_geometry* g, double wave_num, const double* prop, int pol, int kind,
                      double waist, const double* center, double* einc);
/* The same with the beam frame (prop_p, ex_p = the polarisation vector, ey_p
 * = ex rotated by +90 degrees about prop: -pol2 for polarisation 1, pol1 for
 * polarisation 2) and the centre in the particle frame (DDA/Beam.cpp:
 * 198-205). */
int dda_einc_gaussian_frame(const dda_geometry* g, double wave_num, const double* prop_p, const double* ex_p,
                            const double* ey_p, int kind, double waist, const double* center_p, double* einc);

#ifdef __cplusplus
}
#endif

#endif /* DDA_FRONTEND_H */
