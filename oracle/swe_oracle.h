/*
 * swe_oracle.h -- CPU restatement of the reference shallow-water solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA library is
 * checked against; it is never linked into, loaded by, or called from the
 * product path.  Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference leg of bench.py may load it.
 *
 * It restates, loop for loop and operand for operand, the FP64 arithmetic of
 *   src/swe.mjs       (ShallowWater, hllc, flux1D, limiters, boundaries, sponge)
 *   src/geometry.mjs  (cartesianGeometry, sphericalGeometry, cosLat, ...)
 *   src/tide.mjs:103-107 (Tide.eta, as a constituent table)
 * of Syntaxswine/water-simulator.  Compile with -O2 -ffp-contract=off and no
 * fast-math so every + - * / sqrt rounds exactly as the JavaScript engine does.
 *
 * Pinning: the reference is JavaScript and no JS engine exists where this is
 * built, so the oracle is pinned against the reference's own recorded numbers
 * (tools/sphere-baseline.json, the positivity identity at
 * tools/verify-physics.mjs:539, the README accuracy table), see tests/.
 */
#ifndef SWE_ORACLE_H
#define SWE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Same field layout as swe_options in include/swe_b200.h (defaults from
 * src/swe.mjs:170-174 and src/geometry.mjs:190-192). */
typedef struct oracle_options {
  int nx, ny;
  double dx, dy;
  double manning, min_depth, cfl, coriolis;
  int order, limiter, sphere;
  double R, lat0, lat1, omega;
} oracle_options;

typedef struct oracle_sim oracle_sim;

/* field ids (match SWE_FIELD_* of the product header) */
enum { OF_B = 0, OF_H, OF_HU, OF_HV, OF_H0, OF_HU0, OF_HV0, OF_RH, OF_RHU, OF_RHV,
       OF_THETA, OF_MANNING, OF_UU, OF_VV, OF_NFIELDS };
/* geometry row ids (match SWE_GEOM_*) */
enum { OG_DXROW = 0, OG_DYROWN, OG_DYROWS, OG_DYCFL, OG_AREA, OG_LX, OG_LYN, OG_LYS,
       OG_BEDPHI, OG_PHIC, OG_TANPHI, OG_FROW, OG_GEOCOEF, OG_NROWS };
/* boundary kinds / sides (match SWE_BC_*, SWE_SIDE_*) */
enum { OB_REFLECT = 0, OB_OUTFLOW = 1, OB_PERIODIC = 2, OB_FLATHER = 3 };

int          oracle_create(const oracle_options* o, const double* b, const double* h, oracle_sim** out);
void         oracle_destroy(oracle_sim* s);
const char*  oracle_last_error(void);
double*      oracle_field(oracle_sim* s, int field);      /* direct pointer, N doubles (manning: NULL if unset) */
double*      oracle_geom(oracle_sim* s, int row);         /* direct pointer, H doubles */
/* scalars: 0 dx 1 dy 2 R 3 dlam 4 dphi 5 totalArea 6 t 7 steps 8 massFloored 9 eps4 10 lat0 11 lat1 12 omega */
double       oracle_get_scalar(oracle_sim* s, int which);
void         oracle_set_scalar(oracle_sim* s, int which, double v);
void         oracle_set_threads(oracle_sim* s, int threads);

int          oracle_set_boundary(oracle_sim* s, int side, int kind);
/* Flather external values for the next applyBC (value mode) */
int          oracle_set_flather_values(oracle_sim* s, int side, double eta_ext, double u_ext);
/* Flather from a harmonic table: eta = msl + sum amp*cos(omega*t - phase_deg*PI/180), u = u_coef*eta */
int          oracle_set_flather_tide(oracle_sim* s, int side, double msl, int n, const double* amp,
                                     const double* omega, const double* phase_deg, double u_coef);
int          oracle_set_manning_field(oracle_sim* s, const double* n);   /* NULL clears */
int          oracle_set_sponge(oracle_sim* s, int side, int width, double strength, double eta_ref);
int          oracle_clear_sponge(oracle_sim* s);

void         oracle_apply_bc(oracle_sim* s);
void         oracle_residual(oracle_sim* s, double dt);
double       oracle_max_dt(oracle_sim* s);
void         oracle_apply_friction(oracle_sim* s, double dt);
double       oracle_dry_clean(oracle_sim* s);
double       oracle_step(oracle_sim* s, double dt);       /* returns dt taken, 0 on a bad dt */
double       oracle_step_auto(oracle_sim* s);             /* step() with no argument */
double       oracle_volume(oracle_sim* s);
double       oracle_energy(oracle_sim* s);
double       oracle_max_surface_deviation(oracle_sim* s, double ref);
double       oracle_max_speed(oracle_sim* s);
int          oracle_finite(oracle_sim* s);
double       oracle_vel(oracle_sim* s, double hq, double h);
void         oracle_hllc(double* out3, double hL, double huL, double hvL, double hR, double huR,
                         double hvR, double dry);

/* Tangent-linear model of the gauge misfit (see swe_oracle.cpp). */
int          oracle_tlm_misfit(const oracle_options* o, const double* b, const double* eta0, const double* n,
                               const double* db, const double* dn, int ng, const int* gauges, int steps,
                               const double* obs, int threads, double* J, double* dJ, double* dts);
/* A Flather side's tide (src/tide.mjs:103-107): eta(t) = msl + sum amp cos(omega t - phase), u = u_coef eta. */
typedef struct {
  int n;                        /* constituents; 0: the side keeps its constant exterior state */
  double msl, u_coef;
  const double* amp; const double* omega; const double* phase_deg;
} oracle_tide_spec;
/* The same with a boundary kind per side (W, E, S, N; NULL: reflect), the
 * constant Flather exterior surface and normal velocity (NULL: 0), and a
 * tide per side (NULL, or n = 0: none). */
int          oracle_tlm_misfit_bc(const oracle_options* o, const double* b, const double* eta0, const double* n,
                                  const double* db, const double* dn, int ng, const int* gauges, int steps,
                                  const double* obs, int threads, const int* kinds, const double* fl_eta,
                                  const double* fl_u, const oracle_tide_spec* tides, double* J, double* dJ,
                                  double* dts);

#ifdef __cplusplus
}
#endif
#endif
