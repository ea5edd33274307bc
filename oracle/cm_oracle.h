/*
 * cm_oracle.h -- CPU restatement of CudaMONSEL's electron-transport hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA engine is compared
 * against; the library never links, loads or calls it.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * Everything here is plain C99 in double precision and SI units (J, m, 1/m),
 * as the reference computes.  Each function cites the reference source it
 * follows (paths relative to CudaMONSEL/CudaMONSEL/gov/nist/).  The
 * restatement is pinned against golden vectors dumped from the reference
 * itself (oracle/build_ref.py + oracle/ref_driver.cpp -> tests/golden/).
 */
#ifndef CM_ORACLE_H
#define CM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cmo_scene cmo_scene;

/* ---- deviate source: a fixed array (per-function checks) or a seeded generator */
typedef struct {
   const double* fixed;   /* if non-NULL, deviates are taken from here in order */
   int nfixed;
   int used;              /* number of deviates drawn so far */
   uint64_t s[4];         /* xoshiro256** state when fixed == NULL */
} cmo_rng;

void cmo_rng_seed(cmo_rng* r, uint64_t seed);
double cmo_uniform(cmo_rng* r);

/* ---- interpolation (JMONSELutils/ULagrangeInterpolation.cu, NULagrangeInterpolation.cu) */
double cmo_ulagrange_d1(const double* f, int len, double x0, double xinc, int order, double x);
double cmo_ulagrange_d2(const double* f, int n0, int n1, const double x0[2], const double xinc[2], int order,
                        const double x[2]);
void cmo_nu_locate(double x, const double* xs, int n, int order, int out[2]);
double cmo_nu_d1(const double* f, int n, const double* xs, int order, double x);

/* ---- scene construction (SI units) */
cmo_scene* cmo_scene_new(void);
void cmo_scene_free(cmo_scene* s);
/* options: bit 0 = JMONSEL fixes (refraction in ExpQMBarrierSM, proper d3 abscissae) */
void cmo_scene_set_options(cmo_scene* s, int options);
int cmo_add_mott_element(cmo_scene* s, int Z, const double* spwem61, const double* x1_61x201);
int cmo_add_table_file(cmo_scene* s, const char* path);
int cmo_add_material(cmo_scene* s, int nel, const int* Z, const double* atomicWeight, const double* weightFraction,
                     double density, double workfunction, double energyCBbottom, double bandgap, int ncore,
                     const double* coreEnergies);
int cmo_add_msm(cmo_scene* s, int material);
int cmo_msm_add_nistmott(cmo_scene* s, int msm, int method);
int cmo_msm_add_tabulated(cmo_scene* s, int msm, int methodSE, double energyOffset, const int tables[4]);
int cmo_msm_add_fitted(cmo_scene* s, int msm, double energySEgen, double breakE);
int cmo_msm_add_phonon(cmo_scene* s, int msm, double ratemult, double phononE, double temperature, double eps0,
                       double epsInf);
int cmo_msm_add_polaron(cmo_scene* s, int msm, double prefactor, double extinction);
int cmo_msm_set_csd_jln(cmo_scene* s, int msm, double breakE);
int cmo_msm_set_min_e(cmo_scene* s, int msm, double minE);
int cmo_msm_set_barrier(cmo_scene* s, int msm, int classical, double lambda);
int cmo_shape_sphere(cmo_scene* s, const double center[3], double radius);
int cmo_shape_planes(cmo_scene* s, int n, const double* normals, const double* points);
int cmo_shape_intersection(cmo_scene* s, int a, int b);
int cmo_shape_cylinder(cmo_scene* s, const double end0[3], const double end1[3], double radius);
int cmo_shape_union(cmo_scene* s, int a, int b);
int cmo_shape_translate(cmo_scene* s, int shape, const double d[3]);
int cmo_shape_rotate(cmo_scene* s, int shape, const double pivot[3], double phi, double theta, double psi);
int cmo_shape_line(cmo_scene* s, double topz, double width, double length, double thetal, double thetar, double radl,
                   double radr);
int cmo_region(cmo_scene* s, int parent, int msm, int shape);

/* ---- per-function evaluation on arrays, deviates injected (u arrays are row-major) */
void cmo_eval_nistmott(cmo_scene* s, int Z, int n, const double* E, const double* u, double* sigma, double* theta,
                       int* ndev);
/* the same for NISTMottRS method 1, 2 or 3 (JMONSEL/NISTMottRS.cu:76-91 sets each method's constants) */
void cmo_eval_nistmott_method(cmo_scene* s, int Z, int method, int n, const double* E, const double* u, double* sigma,
                              double* theta, int* ndev);
void cmo_eval_table(cmo_scene* s, int table, int n, const double* x3, int order, double* out);
void cmo_eval_tabulated(cmo_scene* s, int msm, int mech, int n, const double* in /* E th ph u0..u5 */,
                        double* out /* rate E th ph hasSE ESE thSE phSE ndev */);
/* the same with stride >= 10 also writes the sampled PE deflection theta in column 9 */
void cmo_eval_tabulated_stride(cmo_scene* s, int msm, int mech, int n, const double* in, double* out, int stride);
/* first index of the 4-point window NULagrangeInterpolation::locate picks on a table's first axis */
int cmo_table_window(cmo_scene* s, int table, double x0);
void cmo_table_locate(cmo_scene* s, int table, int n, const double* x3, int order, int* out /* [6n] */);
void cmo_eval_pick(cmo_scene* s, int msm, int n, const double* in /* E u */, double* out /* index total */);
void cmo_eval_elastic(cmo_scene* s, int msm, int mech, int n, const double* in /* E th ph u0..u3 */,
                      double* out /* rate th ph Z ndev */);
void cmo_eval_pmma(cmo_scene* s, int msm, int n, const double* in /* E len */, double* out /* csd fittedRate polaronRate */);
void cmo_eval_phonon(cmo_scene* s, int msm, int mech, int n, const double* in /* E th ph u0 u1 */,
                     double* out /* rate E th ph Eprev ndev */);
void cmo_eval_shape(cmo_scene* s, int shape, int n, const double* p01,
                    double* out /* nx ny nz u contains(p0) contains(p0,p1) */);
void cmo_eval_barrier(cmo_scene* s, int from_region, int to_region, int struck_shape, int n,
                      const double* in /* E th ph x y z */, double* out /* E th ph x y z region */);
void cmo_eval_freepath(cmo_scene* s, int msm, int n, const double* in /* E u */, double* out);
void cmo_eval_beam(int n, const double* in /* width cx cy cz u0 u1 */, double* out /* x y z */);
int cmo_hist_bin(double min, double max, int nbins, double v);

/* ---- whole trajectories, MonteCarloSS::runMultipleTrajectories with BackscatterStats attached */
typedef struct {
   int64_t back[1026];    /* BackscatterStats back-energy histogram incl. under/overflow: index = bin + 1 */
   int64_t fwd[1026];
   int64_t trajectories;
   int64_t scatter_events, barrier_events, secondaries;
   int64_t dropped_overrange; /* escapes whose bin index falls past the overflow slot (reference writes out of bounds) */
   int64_t elevation[182];    /* BackscatterStats elevation histogram, Histogram(0, pi, 180), index = bin + 1 */
   int64_t azimuth[362];      /* BackscatterStats azimuthal histogram, Histogram(0, 2 pi, 360), index = bin + 1 */
} cmo_tally;

int cmo_run(cmo_scene* s, int chamber_region, double beam_width, double beam_energy, const double center[3],
            int nprim, uint64_t seed, int nbins, cmo_tally* out);

#ifdef __cplusplus
}
#endif
#endif
