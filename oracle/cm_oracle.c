/*
 * cm_oracle.c -- CPU restatement of CudaMONSEL's electron-transport hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see cm_oracle.h).  Plain C99, double precision,
 * SI units, same operation order as the reference so that results agree to
 * the last bit where the reference's own arithmetic is deterministic.
 * Reference paths are relative to CudaMONSEL/CudaMONSEL/gov/nist/.
 */
#include "cm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- constants */
/* microanalysis/EPQLibrary/PhysicalConstants.cu:4-28, Utility/Math2.cu:7 */
#define PI 3.14159265358979323846
static const double AVOGADRO = 6.0221415e23;
static const double BOHR = 5.291772083e-11;
static const double BOLTZMANN = 1.3806505e-23;
static const double ELECTRON_MASS = 9.1093826e-31;
static const double HBAR = 1.05457266e-34;
/* EPQLibrary/ToSI.cu:6-8, FromSI.cu:6-7 */
static const double TOSI_EV = 1.60217653e-19;
#define TOSI_KEV (1.60217653e-19 * 1.0e3)
#define FROMSI_EV (1.0 / 1.60217653e-19)
#define FROMSI_KEV (1.0 / (1.60217653e-19 * 1.0e3))
/* NISTMonte/MonteCarloSS.cu:32-33 */
static const double CHAMBER_RADIUS = 0.1;
static const double SMALL_DISP = 1.0e-15;

#define MAXEL 8
#define MAXMECH 8
#define MAXPLANES 16
#define MAXCHILD 1024

/* ---------------------------------------------------------------- deviates */
static uint64_t splitmix64(uint64_t* x)
{
   uint64_t z = (*x += 0x9e3779b97f4a7c15ULL);
   z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
   z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
   return z ^ (z >> 31);
}

void cmo_rng_seed(cmo_rng* r, uint64_t seed)
{
   memset(r, 0, sizeof(*r));
   for (int i = 0; i < 4; ++i) r->s[i] = splitmix64(&seed);
}

static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* Math2::random() (Utility/Math2.cu:1328-1331) is rand()/RAND_MAX; here either a
 * fixed deviate or xoshiro256** in [0,1). */
double cmo_uniform(cmo_rng* r)
{
   r->used++;
   if (r->fixed) {
      if (r->used - 1 < r->nfixed) return r->fixed[r->used - 1];
      return 0.5;
   }
   uint64_t* s = r->s;
   uint64_t res = rotl(s[1] * 5, 7) * 9;
   uint64_t t = s[1] << 17;
   s[2] ^= s[0];
   s[3] ^= s[1];
   s[1] ^= s[2];
   s[0] ^= s[3];
   s[2] ^= t;
   s[3] = rotl(s[3], 45);
   return (double)(res >> 11) * (1.0 / 9007199254740992.0);
}

/* ---------------------------------------------------------------- uniform-grid Lagrange */
/* JMONSELutils/ULagrangeInterpolation.cu:5-33 */
static double uneville(const double* f, int offset, int order, double x)
{
   int ns = (int)round(x);
   if (ns < 0) ns = 0;
   else if (ns > order) ns = order;
   double c[8], d[8];
   memcpy(c, f + offset, (order + 1) * sizeof(double));
   memcpy(d, f + offset, (order + 1) * sizeof(double));
   double y = c[ns--];
   double ho, hp, w, dy = 0;
   for (int m = 1; m <= order; m++) {
      for (int i = 0; i <= order - m; i++) {
         ho = i - x;
         hp = i + m - x;
         w = c[i + 1] - d[i];
         d[i] = -hp * w / m;
         c[i] = -ho * w / m;
      }
      dy = (2 * ns < (order - 1 - m)) ? c[ns + 1] : d[ns--];
      y += dy;
   }
   return y;
}

/* ULagrangeInterpolation.cu:35-48 */
double cmo_ulagrange_d1(const double* f, int len, double x0, double xinc, int order, double x)
{
   const double reducedx = (x - x0) / xinc;
   int index0 = (int)reducedx - order / 2;
   if (index0 < 0) index0 = 0;
   else if (index0 > len - order - 1) index0 = len - order - 1;
   return uneville(f, index0, order, reducedx - index0);
}

/* ULagrangeInterpolation.cu:80-103 (f row-major [n0][n1]) */
double cmo_ulagrange_d2(const double* f, int n0, int n1, const double x0[2], const double xinc[2], int order,
                        const double x[2])
{
   const double reducedx1 = (x[0] - x0[0]) / xinc[0];
   int index0 = (int)reducedx1 - order / 2;
   if (index0 < 0) index0 = 0;
   else if (index0 > n0 - order - 1) index0 = n0 - order - 1;
   double y[8];
   for (int i = 0; i <= order; i++) y[i] = cmo_ulagrange_d1(f + (size_t)(index0 + i) * n1, n1, x0[1], xinc[1], order, x[1]);
   return cmo_ulagrange_d1(y, order + 1, x0[0] + index0 * xinc[0], xinc[0], order, x[0]);
}

/* ---------------------------------------------------------------- non-uniform Lagrange */
/* JMONSELutils/NULagrangeInterpolation.cu:5-68 */
void cmo_nu_locate(double x, const double* xsamp, int xsamplen, int order, int out[2])
{
   int lowlim = -1;
   int uplim = xsamplen;
   int maxindex = uplim - 1;
   int midpoint, nindex;
   int ascending = xsamp[maxindex] > xsamp[0];
   while ((uplim - lowlim) > 1) {
      midpoint = (uplim + lowlim) >> 1;
      if ((x > xsamp[midpoint]) == ascending) lowlim = midpoint;
      else uplim = midpoint;
   }
   if (lowlim < 0) { out[0] = 0; out[1] = 0; return; }
   if (uplim > maxindex) { out[0] = maxindex - order; out[1] = maxindex; return; }
   if (ascending) nindex = ((x - xsamp[lowlim]) <= (xsamp[uplim] - x)) ? lowlim : uplim;
   else nindex = ((xsamp[lowlim] - x) <= (x - xsamp[uplim])) ? lowlim : uplim;
   int firstInd = lowlim, lastInd = uplim;
   while (((lastInd - firstInd) < order) && (firstInd > 0) && (lastInd < maxindex))
      if (((((xsamp[lowlim] - xsamp[firstInd - 1]) + xsamp[uplim]) - xsamp[lastInd + 1]) >= 0) == ascending) lastInd += 1;
      else firstInd -= 1;
   if (lastInd >= maxindex) { out[0] = maxindex - order; out[1] = nindex; return; }
   if (firstInd <= 0) { out[0] = 0; out[1] = nindex; return; }
   out[0] = firstInd;
   out[1] = nindex;
}

/* NULagrangeInterpolation.cu:85-112 */
static double nu_neville(const double* f, const double* xsamp, const int loc[2], int order, double x)
{
   int offset = loc[0];
   int ns = loc[1] - offset;
   double c[8], d[8];
   memcpy(c, f + offset, (order + 1) * sizeof(double));
   memcpy(d, f + offset, (order + 1) * sizeof(double));
   double y = c[ns--];
   double ho, hp, w, den, dy = 0;
   for (int m = 1; m <= order; m++) {
      for (int i = 0; i <= (order - m); i++) {
         ho = xsamp[i + offset] - x;
         hp = xsamp[i + m + offset] - x;
         w = c[i + 1] - d[i];
         den = ho - hp;
         den = w / den;
         d[i] = hp * den;
         c[i] = ho * den;
      }
      dy = ((2 * ns) < (order - 1 - m)) ? c[ns + 1] : d[ns--];
      y += dy;
   }
   return y;
}

/* NULagrangeInterpolation.cu:131-147 */
double cmo_nu_d1(const double* f, int n, const double* xs, int order, double x)
{
   int loc[2];
   cmo_nu_locate(x, xs, n, order, loc);
   return nu_neville(f, xs, loc, order, x);
}

typedef struct {
   int dim;
   int n[4];
   double* x[4];
   double* v;        /* last index fastest */
   double domain[4][2];
   double range[2];
} nu_table;

/* NULagrangeInterpolation.cu:169-192; f row-major [n0][n1] */
static double nu_d2(const double* f, const int* n, double* const* xs, int order, const double* x)
{
   int loc[2];
   cmo_nu_locate(x[0], xs[0], n[0], order, loc);
   int index0 = loc[0];
   double y[8];
   for (int i = 0; i <= order; i++) y[i] = cmo_nu_d1(f + (size_t)(index0 + i) * n[1], n[1], xs[1], order, x[1]);
   return cmo_nu_d1(y, order + 1, xs[0] + index0, order, x[0]);
}

/* NULagrangeInterpolation.cu:215-240.  The reference interpolates the final
 * 1-D step on xsamp[0][0..order] rather than xsamp[0][index0..index0+order]
 * (line 236); fixes=1 uses the window the values belong to. */
static double nu_d3(const double* f, const int* n, double* const* xs, int order, const double* x, int fixes)
{
   int loc[2];
   cmo_nu_locate(x[0], xs[0], n[0], order, loc);
   int index0 = loc[0];
   double y[8];
   for (int i = 0; i <= order; i++) y[i] = nu_d2(f + (size_t)(index0 + i) * n[1] * n[2], n + 1, xs + 1, order, x + 1);
   return cmo_nu_d1(y, order + 1, fixes ? xs[0] + index0 : xs[0], order, x[0]);
}

/* JMONSEL/NUTableInterpolation.cu:98-115 */
static double table_interp(const nu_table* t, const double* x, int order, int fixes)
{
   switch (t->dim) {
   case 1: return cmo_nu_d1(t->v, t->n[0], t->x[0], order, x[0]);
   case 2: return nu_d2(t->v, t->n, t->x, order, x);
   case 3: return nu_d3(t->v, t->n, t->x, order, x, fixes);
   default: return NAN;
   }
}

/* NUTableInterpolation.cu:117-228 (whitespace-separated text; 1 <= dim <= 3 here) */
static int table_read(const char* path, nu_table* t)
{
   FILE* fp = fopen(path, "r");
   if (!fp) return -1;
   memset(t, 0, sizeof(*t));
   t->range[0] = INFINITY;
   t->range[1] = -INFINITY;
   if (fscanf(fp, "%d", &t->dim) != 1 || t->dim < 1 || t->dim > 3) { fclose(fp); return -2; }
   size_t total = 1;
   for (int i = 0; i < t->dim; i++) {
      if (fscanf(fp, "%d", &t->n[i]) != 1 || t->n[i] < 2) { fclose(fp); return -3; }
      t->x[i] = (double*)malloc(sizeof(double) * t->n[i]);
      for (int j = 0; j < t->n[i]; j++)
         if (fscanf(fp, "%lf", &t->x[i][j]) != 1) { fclose(fp); return -4; }
      if (t->x[i][0] < t->x[i][t->n[i] - 1]) {
         t->domain[i][0] = t->x[i][0];
         t->domain[i][1] = t->x[i][t->n[i] - 1];
      }
      else {
         t->domain[i][1] = t->x[i][0];
         t->domain[i][0] = t->x[i][t->n[i] - 1];
      }
      total *= (size_t)t->n[i];
   }
   t->v = (double*)malloc(sizeof(double) * total);
   for (size_t k = 0; k < total; k++) {
      if (fscanf(fp, "%lf", &t->v[k]) != 1) { fclose(fp); return -5; }
      /* the reference updates range with if / else-if (NUTableInterpolation.cu:169-172) */
      if (t->v[k] < t->range[0]) t->range[0] = t->v[k];
      else if (t->v[k] > t->range[1]) t->range[1] = t->v[k];
   }
   fclose(fp);
   return 0;
}

/* ---------------------------------------------------------------- elastic cross sections */
typedef struct {
   int Z;
   double spwem[61];
   double* x1; /* [61][201] */
   /* NISTMottRS members (JMONSEL/NISTMottRS.cu:76-91), indexed by method 1..3 */
   double extrapolateBelowEnergy[4], mottXSatMin[4], sfBrowning[4];
   /* BrowningEmpiricalCrossSection.cu:11-17 */
   double zp17, zp2, zp3;
} mott_elem;

static const double MAX_NISTMOTT_() { return 20.0 * TOSI_KEV; }

/* EPQLibrary/BrowningEmpiricalCrossSection.cu:24-29 */
static double browning_sigma(const mott_elem* m, double energy)
{
   const double e = energy * FROMSI_KEV;
   const double re = sqrt(e);
   return 3.0e-22 * m->zp17 / (e + 0.005 * m->zp17 * re + 0.0007 * m->zp2 / re);
}

/* BrowningEmpiricalCrossSection.cu:31-45.  The reference's instances hold
 * `const Element& mElement` bound to a temporary Element built from an int
 * (BrowningEmpiricalCrossSection.cu:47-..., .cuh:20), so z is read through a
 * dangling reference.  The compiled reference reads 0 there (every golden
 * Browning angle is consistent with z = 0 and with no other value): r becomes
 * infinite, r1 <= r/(r+1) compares against NaN, and every angle is isotropic.
 * fixes = 1 uses the element's atomic number. */
static double browning_angle(const mott_elem* m, double energy, cmo_rng* r, int fixes)
{
   const double r1 = cmo_uniform(r), r2 = cmo_uniform(r);
   if (!fixes) return acos(1 - 2.0 * r2);
   const double z = m->Z;
   const double e = energy * FROMSI_KEV;
   const double rr = (300.0 * e / z) + (m->zp3 / (3.0e5 * e));
   if (r1 <= rr / (rr + 1)) {
      const double alpha = 7.0e-3 / e;
      return acos(1.0 - ((2.0 * alpha * r2) / (alpha - r2 + 1)));
   }
   return acos(1 - 2.0 * r2);
}

/* EPQLibrary/ScreenedRutherfordScatteringAngle.cu:24-39 */
static double rutherford_sigma(int Z, double energy)
{
   double z = Z;
   double zp = pow(z, 1.0 / 3.0);
   return (7.670843088080456e-38 * zp * (1.0 + z)) / ((energy + ((5.44967975966321e-19 * zp * zp))));
}

static double rutherford_angle(int Z, double energy, cmo_rng* r)
{
   double alpha = (5.44968e-19 * pow(Z, 2.0 / 3.0)) / energy;
   double rr = cmo_uniform(r);
   return acos(1 - 2.0 * alpha * rr / (1 + alpha - rr));
}

static double dl50(void) { return log(0.050 * TOSI_KEV); }
static double param(void) { return (log(20.0 * TOSI_KEV) - dl50()) / 60.0; }

/* JMONSEL/NISTMottRS.cu:103-119: below extrapolateBelowEnergy method 3 is linear in energy, methods 1
 * and 2 scale Browning's cross section */
static double nistmott_sigma(const mott_elem* m, double energy, int method)
{
   if (energy < m->extrapolateBelowEnergy[method]) {
      if (method == 3) return m->mottXSatMin[method] * energy / m->extrapolateBelowEnergy[method];
      return m->sfBrowning[method] * browning_sigma(m, energy);
   }
   if (energy < MAX_NISTMOTT_()) return (BOHR * BOHR) * cmo_ulagrange_d1(m->spwem, 61, dl50(), param(), 3, log(energy));
   return rutherford_sigma(m->Z, energy);
}

/* NISTMottRS.cu:121-154 (Browning's angle below extrapolateBelowEnergy for every method) */
static double nistmott_angle(const mott_elem* m, double energy, int method, cmo_rng* r, int fixes)
{
   if (energy < m->extrapolateBelowEnergy[method]) return browning_angle(m, energy, r, fixes);
   if (energy < MAX_NISTMOTT_()) {
      const double x0[] = { dl50(), 0. };
      const double xinc[] = { param(), 0.005 };
      double lg = log(energy);
      const double x[] = { lg, cmo_uniform(r) };
      const double q = cmo_ulagrange_d2(m->x1, 61, 201, x0, xinc, 3, x);
      const double com = 1.0 - (2.0 * q * q);
      return com > -1.0 ? (com < 1.0 ? acos(com) : 0.0) : PI;
   }
   return rutherford_angle(m->Z, energy, r);
}

static void mott_setup(mott_elem* m)
{
   m->zp17 = pow(m->Z, 1.7);
   m->zp2 = pow(m->Z, 2.0);
   m->zp3 = pow(m->Z, 3.0);
   /* NISTMottRS.cu:82,86-87: 50 eV for method 1, 100 eV for methods 2 and 3; the cross section at the
    * extrapolation energy itself comes from the table branch */
   for (int method = 0; method < 4; ++method) {
      m->extrapolateBelowEnergy[method] = TOSI_EV * (method <= 1 ? 50. : 100.);
      m->mottXSatMin[method] = nistmott_sigma(m, m->extrapolateBelowEnergy[method], method);
      m->sfBrowning[method] = m->mottXSatMin[method] / browning_sigma(m, m->extrapolateBelowEnergy[method]);
   }
}

/* ---------------------------------------------------------------- scene */
typedef struct {
   int nel;
   int Z[MAXEL];
   double A[MAXEL], wf[MAXEL];
   double density, workfunction, ecb, bandgap;
   int ncore;
   double core[16];
} material;

enum { M_NISTMOTT = 1, M_TABULATED, M_FITTED, M_PHONON, M_POLARON };

typedef struct {
   double coef[MAXEL], recipJ[MAXEL], beta[MAXEL];
   double breakE, bh, bhplus1eV, gamma, minE;
   int nce;
} jln_csd;

typedef struct {
   int kind;
   /* elastic: SelectableElasticSM.cu:69-89, NISTMottRS method */
   int nel, method;
   int elem[MAXEL];         /* index into scene mott table */
   double scalefactor[MAXEL];
   double densityNa;
   /* tabulated: TabulatedInelasticSM.cu:461-498 */
   int methodSE;
   double energyOffset, minEgenSE, rateMult;
   int tIIMFP, tRed, tTheta, tSEE0;
   double energyCBbottom, workfunction, bandgap, energyGap, offsetFermiEnergy, bEref;
   int ncore;
   double core[16];
   double eiDomain[2], iimfpDomain[2], rangeSE0[2];
   /* fitted */
   double energySEgen, eFermi;
   jln_csd csd;
   /* phonon */
   double phononE, prefactor;
   /* polaron */
   double extinction, cutoff;
} mechanism;

typedef struct {
   int material;
   int vacuum;
   int nmech;
   mechanism mech[MAXMECH];
   int csd_kind; /* 0 zero, 1 JLN */
   jln_csd csd;
   double minE;
   int classical;
   double lambda, lambdaFactor, u0;
} msm_t;

enum { S_SPHERE = 1, S_PLANES, S_INTERSECTION, S_CYLINDER, S_UNION };

typedef struct {
   int kind;
   double c[3], r;
   int np;
   double n[MAXPLANES][3], p[MAXPLANES][3];
   int a, b;
   /* NormalCylindricalShape: end0, axis = end1 - end0, radius^2, |axis|^2, |axis|, axis / |axis| */
   double e0[3], ax[3], rad2, len2, len, nax[3];
} shape_t;

typedef struct {
   int parent, msm, shape;
   int nchild;
   int child[MAXCHILD];
} region_t;

struct cmo_scene {
   int options;
   mott_elem mott[120];
   int has_mott[120];
   nu_table* tables;
   int ntables;
   material* mats;
   int nmats;
   msm_t* msms;
   int nmsms;
   shape_t* shapes;
   int nshapes;
   region_t* regions;
   int nregions;
};

#define GROW(arr, cnt) arr = realloc(arr, sizeof(*arr) * (size_t)((cnt) + 1)); memset(&arr[cnt], 0, sizeof(*arr))

cmo_scene* cmo_scene_new(void)
{
   cmo_scene* s = (cmo_scene*)calloc(1, sizeof(cmo_scene));
   return s;
}

void cmo_scene_free(cmo_scene* s)
{
   if (!s) return;
   for (int i = 0; i < 120; ++i) free(s->mott[i].x1);
   for (int i = 0; i < s->ntables; ++i) {
      for (int d = 0; d < 4; ++d) free(s->tables[i].x[d]);
      free(s->tables[i].v);
   }
   free(s->tables);
   free(s->mats);
   free(s->msms);
   free(s->shapes);
   free(s->regions);
   free(s);
}

void cmo_scene_set_options(cmo_scene* s, int options) { s->options = options; }

int cmo_add_mott_element(cmo_scene* s, int Z, const double* spwem61, const double* x1)
{
   if (Z < 1 || Z >= 120) return -1;
   mott_elem* m = &s->mott[Z];
   m->Z = Z;
   memcpy(m->spwem, spwem61, sizeof(m->spwem));
   free(m->x1);
   m->x1 = (double*)malloc(sizeof(double) * 61 * 201);
   memcpy(m->x1, x1, sizeof(double) * 61 * 201);
   mott_setup(m);
   s->has_mott[Z] = 1;
   return Z;
}

int cmo_add_table_file(cmo_scene* s, const char* path)
{
   GROW(s->tables, s->ntables);
   if (table_read(path, &s->tables[s->ntables]) != 0) return -1;
   return s->ntables++;
}

int cmo_add_material(cmo_scene* s, int nel, const int* Z, const double* A, const double* wf, double density,
                     double workfunction, double ecb, double bandgap, int ncore, const double* core)
{
   if (nel > MAXEL || ncore > 16) return -1;
   GROW(s->mats, s->nmats);
   material* m = &s->mats[s->nmats];
   m->nel = nel;
   for (int i = 0; i < nel; ++i) {
      m->Z[i] = Z[i];
      m->A[i] = A[i];
      m->wf[i] = wf[i];
   }
   m->density = density;
   m->workfunction = workfunction;
   m->ecb = ecb;
   m->bandgap = bandgap;
   /* SEmaterial keeps core energies in a std::set (sorted ascending, unique) */
   m->ncore = 0;
   for (int i = 0; i < ncore; ++i) {
      double v = core[i];
      int dup = 0, j;
      for (j = 0; j < m->ncore; ++j) if (m->core[j] == v) dup = 1;
      if (dup) continue;
      j = m->ncore++;
      while (j > 0 && m->core[j - 1] > v) { m->core[j] = m->core[j - 1]; --j; }
      m->core[j] = v;
   }
   return s->nmats++;
}

/* SEmaterial::getEFermi (JMONSEL/SEmaterial.cu:201-204) */
static double efermi(const material* m) { return -m->ecb - m->workfunction; }

/* JMONSEL/MONSEL_MaterialScatterModel.cu:13-37 and ExpQMBarrierSM.cu:12-19 */
int cmo_add_msm(cmo_scene* s, int mat)
{
   if (mat < 0 || mat >= s->nmats) return -1;
   GROW(s->msms, s->nmsms);
   msm_t* m = &s->msms[s->nmsms];
   const material* mt = &s->mats[mat];
   m->material = mat;
   m->vacuum = mt->nel == 0;
   if (m->vacuum) m->minE = -INFINITY;
   else {
      m->minE = -mt->ecb;
      if (m->minE < 0.) m->minE = 0.;
   }
   m->classical = 1;
   m->u0 = mt->ecb;
   return s->nmsms++;
}

int cmo_msm_set_barrier(cmo_scene* s, int msm, int classical, double lambda)
{
   msm_t* m = &s->msms[msm];
   m->classical = classical;
   m->lambda = lambda;
   m->lambdaFactor = (PI * lambda * sqrt(ELECTRON_MASS / 2.)) / HBAR;
   return 0;
}

int cmo_msm_set_min_e(cmo_scene* s, int msm, double minE)
{
   s->msms[msm].minE = minE;
   return 0;
}

int cmo_msm_add_nistmott(cmo_scene* s, int msm, int method)
{
   msm_t* m = &s->msms[msm];
   if (m->nmech >= MAXMECH || method < 1 || method > 3) return -1;
   const material* mt = &s->mats[m->material];
   mechanism* k = &m->mech[m->nmech];
   memset(k, 0, sizeof(*k));
   k->kind = M_NISTMOTT;
   k->method = method;
   k->nel = mt->nel;
   k->densityNa = mt->density * AVOGADRO;
   for (int i = 0; i < mt->nel; ++i) {
      if (!s->has_mott[mt->Z[i]]) return -2;
      k->elem[i] = mt->Z[i];
      k->scalefactor[i] = (1000. * mt->wf[i]) / mt->A[i];
   }
   return m->nmech++;
}

int cmo_msm_add_tabulated(cmo_scene* s, int msm, int methodSE, double energyOffset, const int tables[4])
{
   msm_t* m = &s->msms[msm];
   if (m->nmech >= MAXMECH) return -1;
   const material* mt = &s->mats[m->material];
   mechanism* k = &m->mech[m->nmech];
   memset(k, 0, sizeof(*k));
   k->kind = M_TABULATED;
   k->methodSE = (methodSE != 2) && (methodSE != 3) ? 1 : methodSE;
   k->energyOffset = energyOffset;
   k->minEgenSE = 0.;
   k->rateMult = 1.;
   k->tIIMFP = tables[0];
   k->tRed = tables[1];
   k->tTheta = tables[2];
   k->tSEE0 = tables[3];
   k->energyCBbottom = mt->ecb;
   k->workfunction = mt->workfunction;
   k->bandgap = mt->bandgap;
   k->energyGap = k->bandgap;
   k->offsetFermiEnergy = efermi(mt) + energyOffset;
   k->ncore = mt->ncore;
   memcpy(k->core, mt->core, sizeof(k->core));
   k->bEref = k->bandgap > 0. ? -k->bandgap : efermi(mt);
   const nu_table* tr = &s->tables[k->tRed];
   const nu_table* tt = &s->tables[k->tTheta];
   k->eiDomain[0] = tr->domain[0][0];
   k->eiDomain[1] = tr->domain[0][1];
   if (tt->domain[0][0] > k->eiDomain[0]) k->eiDomain[0] = tt->domain[0][0];
   if (tt->domain[0][1] < k->eiDomain[1]) k->eiDomain[1] = tt->domain[0][1];
   k->iimfpDomain[0] = s->tables[k->tIIMFP].domain[0][0];
   k->iimfpDomain[1] = s->tables[k->tIIMFP].domain[0][1];
   if (k->methodSE == 2 || k->methodSE == 3) {
      k->rangeSE0[0] = s->tables[k->tSEE0].range[0];
      k->rangeSE0[1] = s->tables[k->tSEE0].range[1];
   }
   return m->nmech++;
}

/* JMONSEL/JoyLuoNieminenCSD.cu:10-17,35-82 and EPQLibrary/MeanIonizationPotential.cu:43-47,85-89 */
static void jln_init(jln_csd* c, const material* mt, double breakE)
{
   memset(c, 0, sizeof(*c));
   c->breakE = breakE;
   c->bh = -mt->ecb;
   c->nce = mt->nel;
   if (c->nce == 0) return;
   c->bhplus1eV = c->bh + TOSI_EV * 1.;
   if (c->breakE < c->bhplus1eV) c->breakE = c->bhplus1eV;
   for (int i = 0; i < c->nce; ++i) {
      double z = mt->Z[i];
      double J = mt->Z[i] < 13 ? TOSI_EV * (11.5 * z) : TOSI_EV * (9.76 * z + 58.8 * pow(z, -0.19));
      c->recipJ[i] = 1.166 / J;
      c->beta[i] = 1. - (c->recipJ[i] * c->bhplus1eV);
      c->coef[i] = 2.01507E-28 * mt->density * mt->wf[i] * mt->Z[i] / mt->A[i];
   }
   c->minE = c->bh;
   c->gamma = 0.;
   for (int i = 0; i < c->nce; i++) c->gamma += c->coef[i] * log((c->recipJ[i] * c->breakE) + c->beta[i]);
   c->gamma /= pow(c->breakE, 3.5);
}

/* JoyLuoNieminenCSD.cu:91-121 */
static double jln_compute(const jln_csd* c, double len, double kE)
{
   if ((c->nce == 0) || (kE < c->minE) || (kE <= 0.)) return 0.;
   if (kE <= c->breakE) return (kE / pow(1. + (1.5 * c->gamma * len * kE * sqrt(kE)), 2. / 3.)) - kE;
   double loss = 0.;
   for (int i = 0; i < c->nce; i++) loss += c->coef[i] * log((c->recipJ[i] * kE) + c->beta[i]);
   loss *= len / kE;
   if (loss <= (0.1 * kE)) return -loss;
   loss = jln_compute(c, len / 2., kE);
   return loss + jln_compute(c, len / 2., kE + loss);
}

int cmo_msm_set_csd_jln(cmo_scene* s, int msm, double breakE)
{
   msm_t* m = &s->msms[msm];
   m->csd_kind = 1;
   jln_init(&m->csd, &s->mats[m->material], breakE);
   return 0;
}

/* JMONSEL/FittedInelSM.cu:8-33 (its slowing-down algorithm is a JoyLuoNieminenCSD of the material) */
int cmo_msm_add_fitted(cmo_scene* s, int msm, double energySEgen, double breakE)
{
   msm_t* m = &s->msms[msm];
   if (m->nmech >= MAXMECH) return -1;
   mechanism* k = &m->mech[m->nmech];
   memset(k, 0, sizeof(*k));
   k->kind = M_FITTED;
   k->energySEgen = energySEgen;
   k->eFermi = efermi(&s->mats[m->material]);
   jln_init(&k->csd, &s->mats[m->material], breakE);
   return m->nmech++;
}

/* JMONSEL/GanachaudMokraniPhononInelasticSM.cu:8-17 */
int cmo_msm_add_phonon(cmo_scene* s, int msm, double ratemult, double phononE, double temperature, double eps0,
                       double epsInf)
{
   msm_t* m = &s->msms[msm];
   if (m->nmech >= MAXMECH) return -1;
   mechanism* k = &m->mech[m->nmech];
   memset(k, 0, sizeof(*k));
   k->kind = M_PHONON;
   k->phononE = phononE;
   double occ = 0.5 * (1. + (1. / (exp(phononE / (BOLTZMANN * temperature)) - 1.)));
   double epsRatio = (eps0 - epsInf) / eps0 / epsInf;
   k->prefactor = (ratemult * occ * epsRatio) / BOHR;
   return m->nmech++;
}

/* JMONSEL/GanachaudMokraniPolaronTrapSM.cu:8-12 */
int cmo_msm_add_polaron(cmo_scene* s, int msm, double prefactor, double extinction)
{
   msm_t* m = &s->msms[msm];
   if (m->nmech >= MAXMECH) return -1;
   mechanism* k = &m->mech[m->nmech];
   memset(k, 0, sizeof(*k));
   k->kind = M_POLARON;
   k->prefactor = prefactor;
   k->extinction = extinction;
   k->cutoff = -log(10. / prefactor) / extinction;
   return m->nmech++;
}

int cmo_shape_sphere(cmo_scene* s, const double c[3], double r)
{
   GROW(s->shapes, s->nshapes);
   shape_t* sh = &s->shapes[s->nshapes];
   sh->kind = S_SPHERE;
   memcpy(sh->c, c, sizeof(sh->c));
   sh->r = r;
   return s->nshapes++;
}

int cmo_shape_planes(cmo_scene* s, int n, const double* normals, const double* points)
{
   if (n < 1 || n > MAXPLANES) return -1;
   GROW(s->shapes, s->nshapes);
   shape_t* sh = &s->shapes[s->nshapes];
   sh->kind = S_PLANES;
   sh->np = n;
   for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
         sh->n[i][k] = normals[3 * i + k];
         sh->p[i][k] = points[3 * i + k];
      }
   return s->nshapes++;
}

int cmo_shape_intersection(cmo_scene* s, int a, int b)
{
   GROW(s->shapes, s->nshapes);
   shape_t* sh = &s->shapes[s->nshapes];
   sh->kind = S_INTERSECTION;
   sh->a = a;
   sh->b = b;
   return s->nshapes++;
}

/* NormalCylindricalShape(end0, end1, radius) (JMONSEL/NormalCylindricalShape.cu:8-17,
 * NISTMonte/CylindricalShape.cu:11-20).  The members are initialised in their
 * declaration order (NormalCylindricalShape.cuh:29-35), so normalizedaxis is
 * computed from mLen before mLen is set; the compiled reference reads it as 0
 * and gets an axis of infinities (NaN where the axis component is 0), which
 * makes getFirstNormal and contains(p0, p1) never see the cylinder (pinned by
 * the golden vectors).  That is reproduced unless the fixes option is set when
 * the cylinder is created. */
int cmo_shape_cylinder(cmo_scene* s, const double end0[3], const double end1[3], double radius)
{
   GROW(s->shapes, s->nshapes);
   shape_t* sh = &s->shapes[s->nshapes];
   memset(sh, 0, sizeof(*sh));
   sh->kind = S_CYLINDER;
   for (int k = 0; k < 3; ++k) {
      sh->e0[k] = end0[k];
      sh->ax[k] = end1[k] - end0[k];
   }
   sh->rad2 = radius * radius;
   sh->len2 = (sh->ax[0] * sh->ax[0]) + (sh->ax[1] * sh->ax[1]) + (sh->ax[2] * sh->ax[2]);
   sh->len = sqrt(sh->len2);
   const double mlen = (s->options & 1) ? sh->len : 0.0;
   for (int k = 0; k < 3; ++k) sh->nax[k] = sh->ax[k] / mlen;
   return s->nshapes++;
}

/* NormalUnionShape(a, b) (JMONSEL/NormalUnionShape.cu:8-11) */
int cmo_shape_union(cmo_scene* s, int a, int b)
{
   GROW(s->shapes, s->nshapes);
   shape_t* sh = &s->shapes[s->nshapes];
   memset(sh, 0, sizeof(*sh));
   sh->kind = S_UNION;
   sh->a = a;
   sh->b = b;
   return s->nshapes++;
}

/* Plane::translate (NISTMonte/MultiPlaneShape.cu:59-64) applied to every plane;
 * an intersection or union translates both children, a cylinder its end0
 * (NormalCylindricalShape.cu:321-328). */
int cmo_shape_translate(cmo_scene* s, int shape, const double d[3])
{
   shape_t* sh = &s->shapes[shape];
   if (sh->kind == S_PLANES) {
      for (int i = 0; i < sh->np; ++i)
         for (int k = 0; k < 3; ++k) sh->p[i][k] += d[k];
   }
   else if (sh->kind == S_INTERSECTION || sh->kind == S_UNION) {
      cmo_shape_translate(s, sh->a, d);
      cmo_shape_translate(s, sh->b, d);
   }
   else if (sh->kind == S_CYLINDER) {
      for (int k = 0; k < 3; ++k) sh->e0[k] += d[k];
   }
   else if (sh->kind == S_SPHERE) {
      for (int k = 0; k < 3; ++k) sh->c[k] += d[k];
   }
   return 0;
}

/* Transform3D::rotation (Utility/Transform3D.cu:5-40): Euler angles phi about z, theta about y, psi about
 * z, with the reference's separate form for phi == 0 */
static void euler_matrix(double phi, double th, double psi, double r[3][3])
{
   if (phi != 0.0) {
      const double cTh = cos(th), sTh = sin(th), cPhi = cos(phi), sPhi = sin(phi), cPsi = cos(psi), sPsi = sin(psi);
      r[0][0] = cPhi * cTh * cPsi - sPhi * sPsi;
      r[0][1] = -sPhi * cTh * cPsi - cPhi * sPsi;
      r[0][2] = sTh * cPsi;
      r[1][0] = sPhi * cPsi + cPhi * cTh * sPsi;
      r[1][1] = -sPhi * cTh * sPsi + cPhi * cPsi;
      r[1][2] = sTh * sPsi;
      r[2][0] = -cPhi * sTh;
      r[2][1] = sTh * sPhi;
      r[2][2] = cTh;
   }
   else {
      const double cTh = cos(th), sTh = sin(th), cPsi = cos(psi), sPsi = sin(psi);
      r[0][0] = cTh * cPsi;
      r[0][1] = -sPsi;
      r[0][2] = sTh * cPsi;
      r[1][0] = cTh * sPsi;
      r[1][1] = cPsi;
      r[1][2] = sTh * sPsi;
      r[2][0] = -sTh;
      r[2][1] = 0.0;
      r[2][2] = cTh;
   }
}

/* Transform3D::rotate(v, phi, th, psi) (Transform3D.cu:73-92): the matrix times v, each component summed
 * from zero over the columns in order, as its times() does */
static void rot_vec(const double r[3][3], const double v[3], double out[3])
{
   for (int i = 0; i < 3; ++i) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += r[i][k] * v[k];
      out[i] = acc;
   }
}

/* Transform3D::rotate(point, pivot, ...) (Transform3D.cu:125-128): about the pivot */
static void rot_point(const double r[3][3], const double pt[3], const double pivot[3], double out[3])
{
   double d[3], q[3];
   for (int k = 0; k < 3; ++k) d[k] = pt[k] - pivot[k];
   rot_vec(r, d, q);
   for (int k = 0; k < 3; ++k) out[k] = q[k] + pivot[k];
}

/* ITransform::rotate: NormalMultiPlaneShape (NormalMultiPlaneShape.cu:257-261 -> MultiPlaneShape.cu:306-310
 * -> Plane::rotate, MultiPlaneShape.cu:53-57: normal and point), NormalCylindricalShape
 * (NormalCylindricalShape.cu:324-330: end point about the pivot, axis, and the normalised axis from the
 * rotated axis and the length set at construction), Sphere (its centre).  Intersections and unions pass it
 * to their parts (the reference's cast makes that unsafe to run there). */
int cmo_shape_rotate(cmo_scene* s, int shape, const double pivot[3], double phi, double theta, double psi)
{
   double r[3][3];
   euler_matrix(phi, theta, psi, r);
   shape_t* sh = &s->shapes[shape];
   if (sh->kind == S_PLANES) {
      for (int i = 0; i < sh->np; ++i) {
         double n[3], p[3];
         rot_vec(r, sh->n[i], n);
         rot_point(r, sh->p[i], pivot, p);
         memcpy(sh->n[i], n, sizeof(n));
         memcpy(sh->p[i], p, sizeof(p));
      }
   }
   else if (sh->kind == S_INTERSECTION || sh->kind == S_UNION) {
      cmo_shape_rotate(s, sh->a, pivot, phi, theta, psi);
      cmo_shape_rotate(s, sh->b, pivot, phi, theta, psi);
   }
   else if (sh->kind == S_CYLINDER) {
      double e0[3], ax[3];
      rot_point(r, sh->e0, pivot, e0);
      rot_vec(r, sh->ax, ax);
      memcpy(sh->e0, e0, sizeof(e0));
      memcpy(sh->ax, ax, sizeof(ax));
      const double l = sqrt(sh->len2);
      for (int k = 0; k < 3; ++k) sh->nax[k] = sh->ax[k] / l;
   }
   else if (sh->kind == S_SPHERE) {
      double c[3];
      rot_point(r, sh->c, pivot, c);
      memcpy(sh->c, c, sizeof(c));
   }
   return 0;
}

/* JMONSEL/NShapes.cu:55-149.  With a corner radius the sidewall becomes the
 * union of the sidewall (plus a clipping plane) and a cylinder along y.  The
 * reference builds the left union from the RIGHT sidewall's plane set
 * (NShapes.cu:140); that is reproduced unless the fixes option is set when the
 * line is created. */
int cmo_shape_line(cmo_scene* s, double topz, double width, double length, double thetal, double thetar, double radl,
                   double radr)
{
   if (radr < 0.) radr = 0.;
   if (radl < 0.) radl = 0.;
   double signz = !topz ? 0 : (topz > 0 ? 1 : -1);
   if (signz == 0.) signz = 1.;
   double en[12] = { 0., 0., signz, 0., 0., -signz, 0., 1., 0., 0., -1., 0. };
   double ep[12] = { 0., 0., topz, 0., 0., 0., 0., length / 2., 0., 0., -length / 2., 0. };
   int enclosure = cmo_shape_planes(s, 4, en, ep);
   const double root2 = sqrt(2.);
   const double absz = signz * topz;
   double costhetar = cos(thetar), sinthetar = sin(thetar);
   double rn[6] = { costhetar, 0., signz * sinthetar }, rp[6] = { width / 2, 0., 0. };
   int nright = 1;
   if (radr > 0) {
      double rad = sqrt(1 - sinthetar);
      rn[3] = rad / root2;
      rn[4] = 0.;
      rn[5] = (signz * costhetar) / root2 / rad;
      rp[3] = ((width / 2.) - (radr / costhetar)) + (((radr - absz) * sinthetar) / costhetar);
      rp[4] = 0.;
      rp[5] = topz;
      nright = 2;
   }
   int rightNMPS = cmo_shape_planes(s, nright, rn, rp);
   int rightSide = rightNMPS;
   if (radr > 0) {
      double xc = ((width / 2.) - (radr / cos(thetar))) + ((radr - absz) * tan(thetar));
      double zc = topz - (signz * radr);
      double e0[3] = { xc, -length / 2., zc }, e1[3] = { xc, length / 2., zc };
      int cyl = cmo_shape_cylinder(s, e0, e1, radr);
      rightSide = cmo_shape_union(s, rightNMPS, cyl);
   }
   double costhetal = cos(thetal), sinthetal = sin(thetal);
   double ln[6] = { -costhetal, 0., signz * sinthetal }, lp[6] = { -width / 2, 0., 0. };
   int nleft = 1;
   if (radl > 0.) {
      double rad = sqrt(1 - sinthetal);
      ln[3] = -rad / root2;
      ln[4] = 0.;
      ln[5] = (signz * costhetal) / root2 / rad;
      lp[3] = ((-width / 2.) + (radl / costhetal)) - (((radl - absz) * sinthetal) / costhetal);
      lp[4] = 0.;
      lp[5] = topz;
      nleft = 2;
   }
   int leftNMPS = cmo_shape_planes(s, nleft, ln, lp);
   int leftSide = leftNMPS;
   if (radl > 0.) {
      double xc = ((width / 2.) - (radl / cos(thetal))) + ((radl - absz) * tan(thetal));
      double zc = topz - (signz * radl);
      double e0[3] = { -xc, -length / 2., zc }, e1[3] = { -xc, length / 2., zc };
      int cyl = cmo_shape_cylinder(s, e0, e1, radl);
      leftSide = cmo_shape_union(s, (s->options & 1) ? leftNMPS : rightNMPS, cyl);
   }
   int nts = cmo_shape_intersection(s, leftSide, rightSide);
   return cmo_shape_intersection(s, nts, enclosure);
}

/* RegionBase.cu:193-200 */
int cmo_region(cmo_scene* s, int parent, int msm, int shape)
{
   GROW(s->regions, s->nregions);
   region_t* r = &s->regions[s->nregions];
   r->parent = parent;
   r->msm = msm;
   r->shape = shape;
   if (parent >= 0) {
      region_t* p = &s->regions[parent];
      if (p->nchild >= MAXCHILD) return -1;
      p->child[p->nchild++] = s->nregions;
   }
   return s->nregions++;
}

/* ---------------------------------------------------------------- geometry */
typedef struct { double v[4]; } nvec;

/* NormalMultiPlaneShape.cu:26-38 */
static int tie_break(const double* n)
{
   if (n[0] < 0.) return 0;
   if (n[0] == 0.) {
      if (n[1] < 0.) return 0;
      if (n[1] == 0.)
         if (n[2] < 0.) return 0;
   }
   return 1;
}

/* NISTMonte/MultiPlaneShape.cu:23-27 */
static int plane_contains(const double* n, const double* pt, const double* p)
{
   return (((p[0] - pt[0]) * n[0] + (p[1] - pt[1]) * n[1] + (p[2] - pt[2]) * n[2]) <= 0.0);
}

/* NormalMultiPlaneShape.cu:40-171 */
static nvec planes_first_normal(const shape_t* sh, const double* pos0, const double* pos1)
{
   double umin = -INFINITY, umax = INFINITY, u;
   int minindex = -1, maxindex = -1;
   nvec result = { { 0., 0., 0., INFINITY } };
   const double delta[] = { pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2] };
   for (int i = 0; i < sh->np; i++) {
      const double* n = sh->n[i];
      const double* c = sh->p[i];
      double pmc[] = { pos0[0] - c[0], pos0[1] - c[1], pos0[2] - c[2] };
      double numerator = (pmc[0] * n[0]) + (pmc[1] * n[1]) + (pmc[2] * n[2]);
      double denominator = (delta[0] * n[0]) + (delta[1] * n[1]) + (delta[2] * n[2]);
      if (denominator == 0) {
         if ((numerator < 0) || ((numerator == 0) && tie_break(n))) continue;
         return result;
      }
      u = -numerator / denominator;
      if (denominator > 0) {
         if (u < umax) {
            if ((u < 0) || (u <= umin)) return result;
            umax = u;
            maxindex = i;
         }
      }
      else if (u > umin) {
         if ((u > 1) || (u >= umax)) return result;
         umin = u;
         minindex = i;
      }
   }
   if (umin > 0) {
      result.v[3] = umin;
      result.v[0] = sh->n[minindex][0];
      result.v[1] = sh->n[minindex][1];
      result.v[2] = sh->n[minindex][2];
      return result;
   }
   if ((umax <= 1) && (umax > 0.)) {
      result.v[3] = umax;
      result.v[0] = sh->n[maxindex][0];
      result.v[1] = sh->n[maxindex][1];
      result.v[2] = sh->n[maxindex][2];
      return result;
   }
   return result;
}

/* NormalMultiPlaneShape.cu:178-204.  delta[1] and delta[2] are never written
 * by the reference (it writes delta[0] three times); they are taken as 0 here. */
static int planes_contains2(const shape_t* sh, const double* pos0, const double* pos1)
{
   int didDelta = 0;
   double delta[3] = { 0., 0., 0. };
   for (int i = 0; i < sh->np; i++) {
      const double* n = sh->n[i];
      const double* c = sh->p[i];
      const double p0c[] = { pos0[0] - c[0], pos0[1] - c[1], pos0[2] - c[2] };
      double p0cdotn = (p0c[0] * n[0]) + (p0c[1] * n[1]) + (p0c[2] * n[2]);
      if (p0cdotn > 0.) return 0;
      if (p0cdotn == 0.) {
         if (!didDelta) {
            delta[0] = pos1[0] - pos0[0];
            delta[0] = pos1[1] - pos0[1];
            delta[0] = pos1[2] - pos0[2];
            didDelta = 1;
         }
         double deltadotn = (delta[0] * n[0]) + (delta[1] * n[1]) + (delta[2] * n[2]);
         if (deltadotn > 0.) return 0;
         if ((deltadotn == 0.) && !tie_break(n)) return 0;
      }
   }
   return 1;
}

static int shape_contains(const cmo_scene* s, int id, const double* p);

/* NormalMultiPlaneShape.cu:230-240, NormalIntersectionShape.cu:9-12, Sphere.cu:11-14 */
static int shape_contains(const cmo_scene* s, int id, const double* p)
{
   const shape_t* sh = &s->shapes[id];
   switch (sh->kind) {
   case S_SPHERE:
      return ((p[0] - sh->c[0]) * (p[0] - sh->c[0]) + (p[1] - sh->c[1]) * (p[1] - sh->c[1]) +
              (p[2] - sh->c[2]) * (p[2] - sh->c[2])) <= sh->r * sh->r;
   case S_PLANES:
      for (int i = 0; i < sh->np; ++i)
         if (!plane_contains(sh->n[i], sh->p[i], p)) return 0;
      return 1;
   case S_INTERSECTION:
      return shape_contains(s, sh->a, p) && shape_contains(s, sh->b, p);
   case S_UNION: /* SumShape::contains (NISTMonte/SumShape.cu:38-44) */
      return shape_contains(s, sh->a, p) || shape_contains(s, sh->b, p);
   case S_CYLINDER: { /* CylindricalShape::contains (NISTMonte/CylindricalShape.cu:31-48) */
      const double u = (sh->ax[0] * (p[0] - sh->e0[0]) + sh->ax[1] * (p[1] - sh->e0[1]) + sh->ax[2] * (p[2] - sh->e0[2])) /
                       sh->len2;
      const double a = p[0] - (sh->e0[0] + u * sh->ax[0]), b = p[1] - (sh->e0[1] + u * sh->ax[1]),
                   c = p[2] - (sh->e0[2] + u * sh->ax[2]);
      return (u >= 0) && (u <= 1.0) && ((a * a + b * b + c * c) <= sh->rad2);
   }
   }
   return 0;
}

/* NormalCylindricalShape::contains(pos0, pos1) (NormalCylindricalShape.cu:24-98) */
static int cylinder_contains2(const shape_t* sh, const double* pos0, const double* pos1)
{
   const double* na = sh->nax;
   const double p0c[] = { pos0[0] - sh->e0[0], pos0[1] - sh->e0[1], pos0[2] - sh->e0[2] };
   const double p0cdotn = (p0c[0] * na[0]) + (p0c[1] * na[1]) + (p0c[2] * na[2]);
   const double p0cSquared = (p0c[0] * p0c[0]) + (p0c[1] * p0c[1]) + (p0c[2] * p0c[2]);
   const double r2 = p0cSquared - (p0cdotn * p0cdotn);
   const int on_end0 = (p0cdotn == 0) && (r2 <= sh->rad2);
   const int on_end1 = (p0cdotn == sh->len) && (r2 <= sh->rad2);
   const int on_cylinder = (r2 == sh->rad2) && (p0cdotn >= 0) && (p0cdotn <= sh->len);
   const double delta[] = { pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2] };
   if (on_end0 || on_end1) {
      const double dd = (delta[0] * na[0]) + (delta[1] * na[1]) + (delta[2] * na[2]);
      if (dd == 0) {
         if (na[0] == 0) return na[1] == 0 ? na[2] > 0 : na[1] > 0;
         return na[0] > 0;
      }
      return on_end0 ? dd > 0 : dd < 0;
   }
   if (on_cylinder) {
      const double nv[] = { p0c[0] - (p0cdotn * na[0]), p0c[1] - (p0cdotn * na[1]), p0c[2] - (p0cdotn * na[2]) };
      return ((nv[0] * delta[0]) + (nv[1] * delta[1]) + (nv[2] * delta[2])) < 0;
   }
   return (r2 < sh->rad2) && (p0cdotn > 0) && (p0cdotn < sh->len);
}

static int shape_contains2(const cmo_scene* s, int id, const double* p0, const double* p1)
{
   const shape_t* sh = &s->shapes[id];
   if (sh->kind == S_PLANES) return planes_contains2(sh, p0, p1);
   if (sh->kind == S_INTERSECTION) return shape_contains2(s, sh->a, p0, p1) && shape_contains2(s, sh->b, p0, p1);
   if (sh->kind == S_UNION) return shape_contains2(s, sh->a, p0, p1) || shape_contains2(s, sh->b, p0, p1);
   if (sh->kind == S_CYLINDER) return cylinder_contains2(sh, p0, p1);
   return shape_contains(s, id, p0);
}

static nvec shape_first_normal(const cmo_scene* s, int id, const double* pos0, const double* pos1);

/* NormalIntersectionShape.cu:19-239 */
static nvec inter_first_normal(const cmo_scene* s, const shape_t* sh, const double* pos0, const double* pos1)
{
   nvec nointersection = { { 0., 0., 0., INFINITY } };
   int adepth, bdepth;
   double u;
   double delta[] = { pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2] };
   nvec nva = shape_first_normal(s, sh->a, pos0, pos1);
   if (nva.v[3] <= 1.) adepth = ((delta[0] * nva.v[0]) + (delta[1] * nva.v[1]) + (delta[2] * nva.v[2])) > 0 ? 1 : 0;
   else {
      if (!shape_contains2(s, sh->a, pos0, pos1)) return nointersection;
      adepth = 1;
   }
   nvec nvb = shape_first_normal(s, sh->b, pos0, pos1);
   if (nvb.v[3] <= 1.) bdepth = ((delta[0] * nvb.v[0]) + (delta[1] * nvb.v[1]) + (delta[2] * nvb.v[2])) > 0 ? 1 : 0;
   else {
      if (!shape_contains2(s, sh->b, pos0, pos1)) return nointersection;
      if (adepth == 1) return nva;
      bdepth = 1;
   }
   int cdepth = adepth + bdepth;
   const double EXTRAU = 1.e-10;
   for (int guard = 0; guard < 100000; ++guard) {
      if (nva.v[3] < nvb.v[3]) {
         if (bdepth == 1) return nva;
         cdepth = cdepth ^ 1;
         u = nva.v[3] + EXTRAU;
         double tmp[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
         nva = shape_first_normal(s, sh->a, tmp, pos1);
         if (nva.v[3] < INFINITY) nva.v[3] = (nva.v[3] * (1. - u)) + u;
         if (nva.v[3] > 1) {
            if (cdepth == 0) return nointersection;
            else return nvb;
         }
         adepth = adepth ^ 1;
      }
      else if (nva.v[3] > nvb.v[3]) {
         if (adepth == 1) return nvb;
         cdepth = cdepth ^ 1;
         u = nvb.v[3] + EXTRAU;
         double tmp[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
         nvb = shape_first_normal(s, sh->b, tmp, pos1);
         if (nvb.v[3] < INFINITY) nvb.v[3] = (nvb.v[3] * (1. - u)) + u;
         if (nvb.v[3] > 1) {
            if (cdepth == 0) return nointersection;
            else return nva;
         }
         bdepth = bdepth ^ 1;
      }
      else {
         int depthchange = (((adepth ^ 1) - adepth) + (bdepth ^ 1)) - bdepth;
         if (depthchange == 0) {
            u = nva.v[3] + EXTRAU;
            double tmp1[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
            nva = shape_first_normal(s, sh->a, tmp1, pos1);
            if (nva.v[3] < INFINITY) nva.v[3] = (nva.v[3] * (1. - u)) + u;
            u = nvb.v[3] + EXTRAU;
            double tmp2[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
            nvb = shape_first_normal(s, sh->b, tmp2, pos1);
            if (nvb.v[3] < INFINITY) nvb.v[3] = (nvb.v[3] * (1. - u)) + u;
            if (nva.v[3] > 1) {
               if (adepth == 0) return nvb;
               else return nointersection;
            }
            if (nvb.v[3] > 1) {
               if (bdepth == 0) return nva;
               else return nointersection;
            }
            adepth = adepth ^ 1;
            bdepth = bdepth ^ 1;
         }
         else {
            nvec r = { { (nva.v[0] + nvb.v[0]) / 2., (nva.v[1] + nvb.v[1]) / 2., (nva.v[2] + nvb.v[2]) / 2., nva.v[3] } };
            return r;
         }
      }
   }
   return nointersection;
}

/* NormalUnionShape.cu:40-269: the crossings of A and B in order along the step,
 * tracking the depth (number of shapes the point is inside); a crossing where the
 * union's depth changes to or from 0 is the union's boundary. */
static nvec union_first_normal(const cmo_scene* s, const shape_t* sh, const double* pos0, const double* pos1)
{
   nvec nointersection = { { 0., 0., 0., INFINITY } };
   int adepth, bdepth;
   double u;
   const double delta[] = { pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2] };
   nvec nva = shape_first_normal(s, sh->a, pos0, pos1);
   if (nva.v[3] <= 1.) adepth = ((delta[0] * nva.v[0]) + (delta[1] * nva.v[1]) + (delta[2] * nva.v[2])) > 0 ? 1 : 0;
   else {
      if (shape_contains2(s, sh->a, pos0, pos1)) return nointersection;
      adepth = 0;
   }
   nvec nvb = shape_first_normal(s, sh->b, pos0, pos1);
   if (nvb.v[3] <= 1.) bdepth = ((delta[0] * nvb.v[0]) + (delta[1] * nvb.v[1]) + (delta[2] * nvb.v[2])) > 0 ? 1 : 0;
   else {
      if (shape_contains2(s, sh->b, pos0, pos1)) return nointersection;
      return nva;
   }
   int cdepth = adepth + bdepth;
   const double EXTRAU = 1.e-10;
   for (int guard = 0; guard < 100000; ++guard) {
      if (nva.v[3] < nvb.v[3]) {
         if (adepth == cdepth) return nva;
         cdepth = (cdepth == 1 ? 2 : 1);
         u = nva.v[3] + EXTRAU;
         double tmp[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
         nva = shape_first_normal(s, sh->a, tmp, pos1);
         if (nva.v[3] < INFINITY) nva.v[3] = (nva.v[3] * (1. - u)) + u;
         if (nva.v[3] > 1) return cdepth == bdepth ? nvb : nointersection;
         adepth = adepth ^ 1;
      }
      else if (nva.v[3] > nvb.v[3]) {
         if (bdepth == cdepth) return nvb;
         cdepth = (cdepth == 1 ? 2 : 1);
         u = nvb.v[3] + EXTRAU;
         double tmp[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
         nvb = shape_first_normal(s, sh->b, tmp, pos1);
         if (nvb.v[3] < INFINITY) nvb.v[3] = (nvb.v[3] * (1. - u)) + u;
         if (nvb.v[3] > 1) return cdepth == adepth ? nva : nointersection;
         bdepth = bdepth ^ 1;
      }
      else {
         int depthchange = (((adepth ^ 1) - adepth) + (bdepth ^ 1)) - bdepth;
         if (depthchange == 0) {
            u = nva.v[3] + EXTRAU;
            double tmp0[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
            nva = shape_first_normal(s, sh->a, tmp0, pos1);
            if (nva.v[3] < INFINITY) nva.v[3] = (nva.v[3] * (1. - u)) + u;
            u = nvb.v[3] + EXTRAU;
            double tmp1[] = { pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2]) };
            nvb = shape_first_normal(s, sh->b, tmp1, pos1);
            if (nvb.v[3] < INFINITY) nvb.v[3] = (nvb.v[3] * (1. - u)) + u;
            if (nva.v[3] > 1) return cdepth != bdepth ? nvb : nointersection;
            if (nvb.v[3] > 1) return cdepth != adepth ? nva : nointersection;
            adepth = adepth ^ 1;
            bdepth = bdepth ^ 1;
         }
         else {
            nvec r = { { (nva.v[0] + nvb.v[0]) / 2., (nva.v[1] + nvb.v[1]) / 2., (nva.v[2] + nvb.v[2]) / 2., nva.v[3] } };
            return r;
         }
      }
   }
   return nointersection;
}

/* NormalCylindricalShape::getFirstNormal (NormalCylindricalShape.cu:111-322) */
static nvec cylinder_first_normal(const shape_t* sh, const double* pos0, const double* pos1)
{
   nvec nv = { { 0., 0., 0., INFINITY } };
   const double* na = sh->nax;
   const double radius2 = sh->rad2, mLen = sh->len, mLen2 = sh->len2;
   const double p0c[] = { pos0[0] - sh->e0[0], pos0[1] - sh->e0[1], pos0[2] - sh->e0[2] };
   const double p0cSquared = (p0c[0] * p0c[0]) + (p0c[1] * p0c[1]) + (p0c[2] * p0c[2]);
   const double delta[] = { pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2] };
   const double p0cdotn = (p0c[0] * na[0]) + (p0c[1] * na[1]) + (p0c[2] * na[2]);
   const double deltadotn = (delta[0] * na[0]) + (delta[1] * na[1]) + (delta[2] * na[2]);
   const double deltadotnSquared = deltadotn * deltadotn;
   const double p0cdotdelta = (delta[0] * p0c[0]) + (delta[1] * p0c[1]) + (delta[2] * p0c[2]);
   const double deltaSquared = (delta[0] * delta[0]) + (delta[1] * delta[1]) + (delta[2] * delta[2]);
   int intersectionnumber = 0;
   double u = 0., u1 = 0., u2 = 0., projection = 0., savedprojection = 0.;
   if (deltadotn != 0.) {
      u1 = -p0cdotn / deltadotn;
      if ((u1 > 0.) && (u1 <= 1.) && ((p0cSquared + (2 * u1 * p0cdotdelta) + (u1 * u1 * deltaSquared)) <= radius2)) {
         nv.v[3] = u1;
         intersectionnumber = 1;
      }
      u2 = u1 + (mLen / deltadotn);
      if ((u2 > 0.) && (u2 <= 1.) && (u2 < nv.v[3]) &&
          (((p0cSquared + (2 * u2 * p0cdotdelta) + (u2 * u2 * deltaSquared) + mLen2) -
            (2 * mLen * (p0cdotn + (u2 * deltadotn)))) <= radius2)) {
         nv.v[3] = u2;
         intersectionnumber = 2;
      }
   }
   if (!(((u1 < 0) && (u2 < 0)) || ((u1 > 1) && (u2 > 1)))) {
      const double r0Squared = p0cSquared - (p0cdotn * p0cdotn);
      const double r1Squared = (r0Squared + (2. * (p0cdotdelta - (p0cdotn * deltadotn))) + deltaSquared) - deltadotnSquared;
      if ((r0Squared > radius2) || (r1Squared > radius2)) {
         const double a = deltaSquared - deltadotnSquared;
         const double minusbover2 = (p0cdotn * deltadotn) - p0cdotdelta;
         double term = (minusbover2 * minusbover2) - (a * (r0Squared - radius2));
         if (term >= 0) {
            term = sqrt(term);
            u = (minusbover2 + term) / a;
            if ((u > 0) && (u <= 1) && (u < nv.v[3])) {
               projection = p0cdotn + (u * deltadotn);
               if ((projection >= 0) && (projection <= mLen)) {
                  nv.v[3] = u;
                  intersectionnumber = 3;
                  savedprojection = projection;
               }
            }
            u = (minusbover2 - term) / a;
            if ((u > 0) && (u <= 1) && (u < nv.v[3])) {
               projection = p0cdotn + (u * deltadotn);
               if ((projection >= 0) && (projection <= mLen)) {
                  nv.v[3] = u;
                  intersectionnumber = 4;
                  savedprojection = projection;
               }
            }
         }
      }
   }
   switch (intersectionnumber) {
   case 1:
      nv.v[0] = -na[0];
      nv.v[1] = -na[1];
      nv.v[2] = -na[2];
      return nv;
   case 2:
      nv.v[0] = na[0];
      nv.v[1] = na[1];
      nv.v[2] = na[2];
      return nv;
   case 3:
   case 4: {
      const double normalv[] = { (p0c[0] + (nv.v[3] * delta[0])) - (savedprojection * na[0]),
                                 (p0c[1] + (nv.v[3] * delta[1])) - (savedprojection * na[1]),
                                 (p0c[2] + (nv.v[3] * delta[2])) - (savedprojection * na[2]) };
      const double normalvmag = sqrt((normalv[0] * normalv[0]) + (normalv[1] * normalv[1]) + (normalv[2] * normalv[2]));
      nv.v[0] = normalv[0] / normalvmag;
      nv.v[1] = normalv[1] / normalvmag;
      nv.v[2] = normalv[2] / normalvmag;
      return nv;
   }
   }
   return nv;
}

/* NISTMonte/Sphere.cu:21-45 (the normal is not defined for a sphere; returned as 0) */
static double sphere_first_intersection(const shape_t* sh, const double* pos0, const double* pos1)
{
   const double d[] = { pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2] };
   const double m[] = { pos0[0] - sh->c[0], pos0[1] - sh->c[1], pos0[2] - sh->c[2] };
   const double ma2 = -2.0 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
   const double b = 2.0 * (m[0] * d[0] + m[1] * d[1] + m[2] * d[2]);
   const double c2 = 2.0 * ((m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) - sh->r * sh->r);
   const double f = b * b + ma2 * c2;
   if (f >= 0) {
      double up = (b + sqrt(f)) / ma2;
      double un = (b - sqrt(f)) / ma2;
      if (up < 0.0) up = INFINITY;
      if (un < 0.0) un = INFINITY;
      return fmin(up, un);
   }
   return INFINITY;
}

static nvec shape_first_normal(const cmo_scene* s, int id, const double* pos0, const double* pos1)
{
   const shape_t* sh = &s->shapes[id];
   if (sh->kind == S_PLANES) return planes_first_normal(sh, pos0, pos1);
   if (sh->kind == S_INTERSECTION) return inter_first_normal(s, sh, pos0, pos1);
   if (sh->kind == S_UNION) return union_first_normal(s, sh, pos0, pos1);
   if (sh->kind == S_CYLINDER) return cylinder_first_normal(sh, pos0, pos1);
   nvec r = { { 0., 0., 0., sphere_first_intersection(sh, pos0, pos1) } };
   return r;
}

/* RegionBase.cu:50-60 */
static int containing_subregion(const cmo_scene* s, int reg, const double* pos)
{
   const region_t* r = &s->regions[reg];
   if (shape_contains(s, r->shape, pos)) {
      for (int i = 0; i < r->nchild; ++i) {
         int c = containing_subregion(s, r->child[i], pos);
         if (c >= 0) return c;
      }
      return reg;
   }
   return -1;
}

static int is_containing_region(const cmo_scene* s, int reg, int target)
{
   const region_t* r = &s->regions[reg];
   for (int i = 0; i < r->nchild; ++i)
      if (r->child[i] == target || is_containing_region(s, r->child[i], target)) return 1;
   return 0;
}

/* RegionBase.cu:74-119.  Returns the next region (-1 = outside the chamber),
 * clips p1 and reports the shape whose boundary was struck and its normal. */
static int find_end_of_step(const cmo_scene* s, int reg, const double* p0, double* p1, nvec* hitnormal)
{
   const region_t* r = &s->regions[reg];
   int base = reg;
   nvec nv = shape_first_normal(s, r->shape, p0, p1);
   double t = nv.v[3];
   *hitnormal = nv;
   if ((t <= 1.0) && r->parent >= 0) base = r->parent;
   int res = reg;
   for (int i = 0; i < r->nchild; ++i) {
      const region_t* sub = &s->regions[r->child[i]];
      nvec cn = shape_first_normal(s, sub->shape, p0, p1);
      double candidate = cn.v[3];
      if ((candidate <= 1.0) && (candidate < t)) {
         t = candidate;
         base = r->child[i];
         *hitnormal = cn;
      }
   }
   if (t <= 1.0) {
      const double delta[] = { p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2] };
      p1[0] = p0[0] + (t * delta[0]);
      p1[1] = p0[1] + (t * delta[1]);
      p1[2] = p0[2] + (t * delta[2]);
      /* Math2::normalize3d / multiply / plus3d */
      double mag = sqrt(delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2]);
      const double over[] = { p1[0] + SMALL_DISP * (delta[0] / mag), p1[1] + SMALL_DISP * (delta[1] / mag),
                              p1[2] + SMALL_DISP * (delta[2] / mag) };
      while (base >= 0) {
         res = containing_subregion(s, base, over);
         if (res >= 0) return res;
         base = s->regions[base].parent;
      }
      return -1;
   }
   return res;
}

/* ---------------------------------------------------------------- electrons */
typedef struct {
   double pos[3];
   double theta, phi, E, Eprev;
   int region;
   int steps;
   int complete;
   nvec hit;       /* normal of the last boundary struck (for the barrier) */
   int hitshape;
} electron;

/* NISTMonte/Electron.cu:100-109 */
static void candidate_point(const electron* e, double dS, double* out)
{
   double st = sin(e->theta);
   out[0] = e->pos[0] + dS * cos(e->phi) * st;
   out[1] = e->pos[1] + dS * sin(e->phi) * st;
   out[2] = e->pos[2] + dS * cos(e->theta);
}

/* Electron.cu:111-131 and TabulatedInelasticSM.cu:68-85 */
static void update_direction(double* theta, double* phi, double dTheta, double dPhi)
{
   double ct = cos(*theta), st = sin(*theta);
   double cp = cos(*phi), sp = sin(*phi);
   double ca = cos(dTheta), sa = sin(dTheta);
   double cb = cos(dPhi);
   double xx = (cb * ct * sa) + (ca * st);
   double yy = sa * sin(dPhi);
   double dx = (cp * xx) - (sp * yy);
   double dy = (cp * yy) + (sp * xx);
   double dz = (ca * ct) - (cb * sa * st);
   *theta = atan2(sqrt((dx * dx) + (dy * dy)), dz);
   *phi = atan2(dy, dx);
}

/* ---------------------------------------------------------------- mechanisms */
/* SelectableElasticSM.cu:25-47 */
static double elastic_set_cache(const cmo_scene* s, const mechanism* k, double kE, double* cum)
{
   double total = 0.;
   for (int i = 0; i < k->nel; i++) {
      total += nistmott_sigma(&s->mott[k->elem[i]], kE, k->method) * k->scalefactor[i];
      cum[i] = total;
   }
   return total;
}

/* TabulatedInelasticSM.cu:436-459 */
static double tabulated_rate(const cmo_scene* s, const mechanism* k, double E)
{
   double kEa = E + k->energyOffset;
   if (kEa < k->iimfpDomain[0]) return 0.;
   return k->rateMult * table_interp(&s->tables[k->tIIMFP], &kEa, 1, s->options & 1);
}

/* GanachaudMokraniPhononInelasticSM.cu:46-72 */
static double phonon_rate(const mechanism* k, double kE)
{
   if (kE < k->phononE) return 0.;
   double x = k->phononE / kE;
   if (x < 0.1) return k->prefactor * x * log(4. / x);
   else if (x >= 1.) return 0.;
   double temp = sqrt(1. - x);
   return k->prefactor * x * log((1. + temp) / (1. - temp));
}

static double mech_rate(const cmo_scene* s, const mechanism* k, const electron* e)
{
   double cum[MAXEL];
   switch (k->kind) {
   case M_NISTMOTT: return elastic_set_cache(s, k, e->E, cum) * k->densityNa;
   case M_TABULATED: return tabulated_rate(s, k, e->E);
   case M_FITTED: /* FittedInelSM.cu:20-25 */
      if (e->E <= (k->energySEgen + k->eFermi)) return 0.;
      return (-jln_compute(&k->csd, 1.e-10, e->E) * 1.e10) / k->energySEgen;
   case M_PHONON: return phonon_rate(k, e->E);
   case M_POLARON: /* GanachaudMokraniPolaronTrapSM.cu:21-27 */
      if (e->E > k->cutoff) return 0.;
      return k->prefactor * exp(-k->extinction * e->E);
   }
   return 0.;
}

/* TabulatedInelasticSM.cu:87-101 */
static void sim_esef(const mechanism* k, double Eq, double deltaE, double r, double* ESEf, double* theta)
{
   double q = sqrt(Eq);
   double kz = (deltaE - Eq) / 2. / q;
   double kzf = kz + q;
   double Ezq = kzf * kzf;
   double minE = (k->offsetFermiEnergy + k->bandgap) - Ezq;
   if (minE < 0.) minE = 0.;
   double maxE = k->offsetFermiEnergy - (kz * kz);
   double Exy = (minE * (1. - r)) + (maxE * r);
   *ESEf = Exy + Ezq;
   *theta = acos(kzf / sqrt(*ESEf));
}

/* TabulatedInelasticSM.cu:153-207 with the constructor defaults (no dispersion, default ratios) */
static double pick_be(const mechanism* k, double Eq, double deltaE)
{
   int i;
   (void)Eq;
   if ((k->ncore > 0) && (deltaE <= k->core[0])) return 0.;
   double energyForIonization = deltaE;
   for (i = 0; (i < k->ncore) && (k->core[i] <= energyForIonization); i++)
      ;
   if (i == 0) return 0.;
   return k->core[i - 1];
}

static double g_last_theta; /* the PE deflection sampled by the last tabulated_scatter (per-function checks) */

/* TabulatedInelasticSM.cu:209-434.  Returns 1 and fills *se when a secondary is made. */
static int tabulated_scatter(const cmo_scene* s, const mechanism* k, electron* pe, electron* se, cmo_rng* r)
{
   g_last_theta = 0.;
   int fixes = s->options & 1;
   double kE0 = pe->E;
   double kE = kE0 + k->energyOffset;
   if (kE < k->eiDomain[0]) return 0;
   double theta = 0., phi = 0.;
   double energySE, thetaSE, phiSE;
   double randoms[4];
   for (int i = 0; i < 4; ++i) randoms[i] = cmo_uniform(r);
   double in[3] = { kE, randoms[0], 0. };
   double deltaE = kE * table_interp(&s->tables[k->tRed], in, 3, fixes);
   if ((deltaE < k->energyGap) && (deltaE > (0.95 * k->energyGap))) deltaE = k->energyGap;
   double theta0PE = pe->theta, phi0PE = pe->phi;
   if (deltaE >= k->bandgap) {
      in[1] = (deltaE - k->energyGap) / (kE - k->offsetFermiEnergy - (2. * k->energyGap));
      if (in[1] > 1.) in[1] = 1.;
      else if (in[1] < 0.) in[1] = 0.;
      in[2] = randoms[1];
      theta = table_interp(&s->tables[k->tTheta], in, 3, fixes);
      g_last_theta = theta;
      phi = 2. * PI * randoms[2];
      update_direction(&pe->theta, &pe->phi, theta, phi);
   }
   pe->E = kE0 - deltaE;
   if (deltaE < k->bandgap) return 0;
   double Eq = (2. * kE) - deltaE - (2. * sqrt(kE * (kE - deltaE)) * cos(theta));
   *se = *pe;
   se->steps = 0;
   se->complete = 0;
   se->Eprev = 0;
   double be;
   switch (k->methodSE) {
   case 1:
      energySE = (deltaE + k->bEref) - pick_be(k, Eq, deltaE);
      if ((energySE + k->energyCBbottom) < k->minEgenSE) return 0;
      thetaSE = PI / 2. - theta;
      phiSE = phi + PI;
      se->theta = theta0PE;
      se->phi = phi0PE;
      update_direction(&se->theta, &se->phi, thetaSE, phiSE);
      break;
   case 2:
      be = pick_be(k, Eq, deltaE);
      if (be > 0.) energySE = (deltaE + k->bEref) - be;
      else {
         double in2[3] = { deltaE, randoms[3], 0. };
         double e0 = table_interp(&s->tables[k->tSEE0], in2, 3, fixes);
         if (e0 < k->rangeSE0[0]) e0 = k->rangeSE0[0];
         else if (e0 > k->rangeSE0[1]) e0 = k->rangeSE0[1];
         energySE = (deltaE + e0) - k->energyOffset;
      }
      if ((energySE + k->energyCBbottom) < k->minEgenSE) return 0;
      thetaSE = PI / 2. - theta;
      phiSE = phi + PI;
      se->theta = theta0PE;
      se->phi = phi0PE;
      update_direction(&se->theta, &se->phi, thetaSE, phiSE);
      break;
   default: /* 3 */
      be = pick_be(k, Eq, deltaE);
      if (be > 0.) {
         energySE = (deltaE + k->bEref) - be;
         if ((energySE + k->energyCBbottom) < k->minEgenSE) return 0;
         thetaSE = acos(1. - (2. * cmo_uniform(r)));
         phiSE = 2. * PI * cmo_uniform(r);
         se->theta = thetaSE;
         se->phi = phiSE;
      }
      else {
         double root = 2. * sqrt(k->offsetFermiEnergy * (k->offsetFermiEnergy + deltaE));
         double sum = (2. * k->offsetFermiEnergy) + deltaE;
         double Eqmin = sum - root, Eqmax = sum + root;
         if ((Eqmin <= Eq) && (Eq <= Eqmax)) {
            double esef, th1;
            sim_esef(k, Eq, deltaE, randoms[3], &esef, &th1);
            energySE = esef - k->energyOffset;
            if ((energySE + k->energyCBbottom) < k->minEgenSE) return 0;
            thetaSE = PI / 2. - theta;
            phiSE = phi + PI;
            double ndt = thetaSE, ndp = phiSE;
            update_direction(&ndt, &ndp, th1, 2. * PI * cmo_uniform(r));
            se->theta = theta0PE;
            se->phi = phi0PE;
            update_direction(&se->theta, &se->phi, ndt, ndp);
         }
         else {
            double in2[3] = { deltaE, randoms[3], 0. };
            double e0 = table_interp(&s->tables[k->tSEE0], in2, 3, fixes);
            if (e0 < k->rangeSE0[0]) e0 = k->rangeSE0[0];
            else if (e0 > k->rangeSE0[1]) e0 = k->rangeSE0[1];
            energySE = (deltaE + e0) - k->energyOffset;
            if ((energySE + k->energyCBbottom) < k->minEgenSE) return 0;
            thetaSE = acos(1. - (2. * cmo_uniform(r)));
            phiSE = 2 * PI * cmo_uniform(r);
            se->theta = thetaSE;
            se->phi = phiSE;
         }
      }
      break;
   }
   se->E = energySE;
   se->Eprev = energySE;
   return 1;
}

/* SelectableElasticSM.cu:49-67 */
static int elastic_scatter(const cmo_scene* s, const mechanism* k, electron* pe, cmo_rng* r, int* Zout)
{
   double cum[MAXEL];
   double kE = pe->Eprev;
   double total = elastic_set_cache(s, k, kE, cum);
   double rr = cmo_uniform(r) * total;
   int index = 0;
   while (cum[index] < rr) index++;
   double alpha = nistmott_angle(&s->mott[k->elem[index]], kE, k->method, r, s->options & 1);
   double beta = 2 * PI * cmo_uniform(r);
   update_direction(&pe->theta, &pe->phi, alpha, beta);
   if (Zout) *Zout = k->elem[index];
   return 0;
}

/* GanachaudMokraniPhononInelasticSM.cu:19-44 */
static void phonon_scatter(const mechanism* k, electron* pe, cmo_rng* r)
{
   double kE0 = pe->E;
   if (kE0 < k->phononE) return;
   double x = k->phononE / kE0;
   double randoms[2];
   randoms[0] = cmo_uniform(r);
   randoms[1] = cmo_uniform(r);
   double costheta;
   if (x < 0.1) costheta = 1 + (((x * x) - (pow(16., randoms[0]) * pow(x, 2. - (2. * randoms[0])))) / 8.);
   else {
      double root = sqrt(1. - x);
      double temp = pow(((-2. * (1 + root)) + x) / ((-2. * (1 - root)) + x), randoms[0]);
      costheta = temp + (((x - 2.) * (temp - 1)) / 2. / root);
   }
   double phi = 2. * PI * randoms[1];
   update_direction(&pe->theta, &pe->phi, acos(costheta), phi);
   pe->E = kE0 - k->phononE;
   pe->Eprev = kE0;
}

/* dispatches ScatterMechanism::scatter; returns 1 if *se holds a new electron */
static int mech_scatter(const cmo_scene* s, const mechanism* k, electron* pe, electron* se, cmo_rng* r)
{
   switch (k->kind) {
   case M_NISTMOTT: return elastic_scatter(s, k, pe, r, NULL);
   case M_TABULATED: return tabulated_scatter(s, k, pe, se, r);
   case M_FITTED: { /* FittedInelSM.cu:13-18 */
      double phi = 2 * PI * cmo_uniform(r);
      double theta = acos(1. - (2. * cmo_uniform(r)));
      *se = *pe;
      se->steps = 0;
      se->complete = 0;
      se->theta = theta;
      se->phi = phi;
      se->E = se->Eprev = k->energySEgen + k->eFermi;
      return 1;
   }
   case M_PHONON: phonon_scatter(k, pe, r); return 0;
   case M_POLARON: /* GanachaudMokraniPolaronTrapSM.cu:14-19 */
      pe->E = 0.;
      pe->complete = 1;
      return 0;
   }
   return 0;
}

/* MONSEL_MaterialScatterModel.cu:44-62 */
static double msm_set_cache(const cmo_scene* s, const msm_t* m, const electron* e, double* cum)
{
   double total = 0.;
   for (int i = 0; i < m->nmech; ++i) {
      total += mech_rate(s, &m->mech[i], e);
      cum[i] = total;
   }
   return total;
}

/* MONSEL_MaterialScatterModel.cu:64-91 */
static double msm_free_path(const cmo_scene* s, const msm_t* m, electron* e, double* cum, double* total, cmo_rng* r)
{
   *total = msm_set_cache(s, m, e, cum);
   double maxFreePath = 2. * CHAMBER_RADIUS;
   if (*total != 0.) {
      double freepath = -log(cmo_uniform(r)) / *total;
      return freepath > maxFreePath ? maxFreePath : freepath;
   }
   if (e->steps > 1000000) e->complete = 1;
   return maxFreePath;
}

/* ExpQMBarrierSM.cu:30-48 */
static double general_barrier_t(const msm_t* m, double rootPerpE, double rootDiff)
{
   double k1 = m->lambdaFactor * rootPerpE;
   if (k1 > 50.) return 1.;
   double k2 = m->lambdaFactor * rootDiff;
   double kplus = k1 + k2, kminus = k1 - k2;
   double ratio = sinh(kminus) / sinh(kplus);
   return 1. - (ratio * ratio);
}

/* ExpQMBarrierSM.cu:50-219.  nb is the struck shape's outward normal when the
 * shape reports one; the reference replaces it by the direction of motion
 * whenever it exists (line 111), which the fixes option corrects. */
static void barrier_scatter(const cmo_scene* s, const msm_t* m, electron* pe, int next, const nvec* struck_normal,
                            int have_normal, cmo_rng* r)
{
   int cur = pe->region;
   if (cur == next) return;
   const material* curmat = &s->mats[s->msms[s->regions[cur].msm].material];
   const material* nextmat = &s->mats[s->msms[s->regions[next].msm].material];
   double deltaU = -curmat->ecb;
   if (!(deltaU == -m->u0)) return;
   deltaU += nextmat->ecb;
   double nb[3] = { 0, 0, 0 };
   if (have_normal) {
      double sign = is_containing_region(s, cur, next) ? -1. : 1.;
      for (int i = 0; i < 3; ++i) nb[i] = struck_normal->v[i] * sign;
   }
   double theta0 = pe->theta, phi0 = pe->phi;
   double sintheta0 = sin(theta0);
   double n0[3] = { sintheta0 * cos(phi0), sintheta0 * sin(phi0), cos(theta0) };
   if (have_normal && !(s->options & 1)) { nb[0] = n0[0]; nb[1] = n0[1]; nb[2] = n0[2]; }
   if (!have_normal) { nb[0] = n0[0]; nb[1] = n0[1]; nb[2] = n0[2]; }
   double cosalpha = (n0[0] * nb[0]) + (n0[1] * nb[1]) + (n0[2] * nb[2]);
   if (cosalpha <= 0.) {
      double p[3] = { pe->pos[0] - (SMALL_DISP * nb[0]), pe->pos[1] - (SMALL_DISP * nb[1]), pe->pos[2] - (SMALL_DISP * nb[2]) };
      memcpy(pe->pos, p, sizeof(p));
      return;
   }
   if (deltaU == 0.) {
      double p[3] = { pe->pos[0] + (SMALL_DISP * nb[0]), pe->pos[1] + (SMALL_DISP * nb[1]), pe->pos[2] + (SMALL_DISP * nb[2]) };
      memcpy(pe->pos, p, sizeof(p));
      pe->region = next;
      return;
   }
   double kE0 = pe->E;
   double perpE = kE0 <= 0. ? 0. : cosalpha * cosalpha * kE0;
   double rootPerpE = 0., rootDiff = 0.;
   int transmits;
   if ((perpE == 0.) || (perpE <= deltaU)) transmits = 0;
   else {
      rootPerpE = sqrt(perpE);
      rootDiff = sqrt(perpE - deltaU);
      if (m->classical) transmits = 1;
      else {
         double tp;
         if (m->lambda == 0.) {
            double ksum = rootPerpE + rootDiff;
            tp = (4. * rootPerpE * rootDiff) / (ksum * ksum);
         }
         else tp = general_barrier_t(m, rootPerpE, rootDiff);
         transmits = cmo_uniform(r) < tp;
      }
   }
   double nf[3];
   if (transmits) {
      double factor = cosalpha * ((rootDiff / rootPerpE) - 1.);
      for (int i = 0; i < 3; i++) nf[i] = n0[i] + (factor * nb[i]);
      nf[2] /= sqrt((nf[0] * nf[0]) + (nf[1] * nf[1]) + (nf[2] * nf[2]));
      pe->E = kE0 - deltaU;
      pe->region = next;
      double p[3] = { pe->pos[0] + (SMALL_DISP * nb[0]), pe->pos[1] + (SMALL_DISP * nb[1]), pe->pos[2] + (SMALL_DISP * nb[2]) };
      memcpy(pe->pos, p, sizeof(p));
   }
   else {
      double twocosalpha = 2. * cosalpha;
      for (int i = 0; i < 3; i++) nf[i] = n0[i] - (nb[i] * twocosalpha);
      double p[3] = { pe->pos[0] - (SMALL_DISP * nb[0]), pe->pos[1] - (SMALL_DISP * nb[1]), pe->pos[2] - (SMALL_DISP * nb[2]) };
      memcpy(pe->pos, p, sizeof(p));
   }
   pe->theta = acos(nf[2]);
   pe->phi = atan2(nf[1], nf[0]);
}

/* ---------------------------------------------------------------- histogram (Utility/Histogram.cu:25-42,73-95) */
typedef struct {
   int nbins;
   double binMin[1025];
} histo;

static void histo_init(histo* h, double min, double max, int nBins)
{
   if (max < min) { double t = min; min = max; max = t; }
   h->nbins = nBins;
   const double delta = (max - min) / nBins;
   h->binMin[0] = min;
   for (int i = 1; i <= nBins; ++i) h->binMin[i] = min + i * delta;
}

/* Amphibian/Algorithm.cu:5-14: returns the match index or the insertion point */
static int histo_bin(const histo* h, double val)
{
   int l = 0, r = h->nbins;
   while (l <= r) {
      int mid = l + (r - l) / 2;
      if (h->binMin[mid] == val) return mid;
      if (h->binMin[mid] < val) l = mid + 1;
      else r = mid - 1;
   }
   return l;
}

int cmo_hist_bin(double min, double max, int nbins, double v)
{
   histo h;
   if (nbins < 1 || nbins > 1024) return -99;
   histo_init(&h, min, max, nbins);
   return histo_bin(&h, v);
}

/* ---------------------------------------------------------------- MonteCarloSS */
#define STACKMAX 4096

typedef struct {
   cmo_scene* s;
   int chamber;
   histo h;
   cmo_tally* t;
   cmo_rng* r;
   histo h_el, h_az; /* BackscatterStats.cu:105-106 */
} run_ctx;

/* BackscatterStats.cu:140-181: elevation and azimuth first, then the energy histogram */
static void tally_escape(run_ctx* c, const electron* e)
{
   const double* pos = e->pos;
   const double elevation = (PI / 2) - atan2(pos[2], sqrt((pos[0] * pos[0]) + (pos[1] * pos[1])));
   double azimuth = atan2(pos[1], pos[0]);
   if (azimuth < 0.0) azimuth = (2.0 * PI) + azimuth;
   const int be = histo_bin(&c->h_el, elevation) + 1, ba = histo_bin(&c->h_az, azimuth) + 1;
   if (be <= 181) c->t->elevation[be]++; /* past the overflow slot the reference writes out of bounds */
   if (ba <= 361) c->t->azimuth[ba]++;
   const double kEeV = e->E * FROMSI_EV;
   int b = histo_bin(&c->h, kEeV) + 1;
   if (b > c->h.nbins + 1) { c->t->dropped_overrange++; return; }
   if (elevation < (PI / 2.0)) c->t->fwd[b]++;
   else c->t->back[b]++;
}

/* MonteCarloSS.cu:107-163 */
static int take_step(run_ctx* c, electron* e, electron* se)
{
   cmo_scene* s = c->s;
   double pos0[3] = { e->pos[0], e->pos[1], e->pos[2] };
   int cur = e->region;
   if (cur < 0 || !shape_contains(s, s->regions[cur].shape, pos0)) {
      cur = containing_subregion(s, c->chamber, pos0);
      e->region = cur;
      if (cur < 0) { e->complete = 1; return 0; }
   }
   const msm_t* m = &s->msms[s->regions[cur].msm];
   double cum[MAXMECH], total;
   double fp = msm_free_path(s, m, e, cum, &total, c->r);
   double pos1[3];
   candidate_point(e, fp, pos1);
   nvec hit;
   int next = find_end_of_step(s, cur, pos0, pos1, &hit);
   double dd = sqrt((pos1[0] - pos0[0]) * (pos1[0] - pos0[0]) + (pos1[1] - pos0[1]) * (pos1[1] - pos0[1]) +
                    (pos1[2] - pos0[2]) * (pos1[2] - pos0[2]));
   double dE = m->csd_kind == 1 ? jln_compute(&m->csd, dd, e->E) : 0.;
   memcpy(e->pos, pos1, sizeof(pos1));
   e->Eprev = e->E;
   e->E += dE;
   e->steps++;
   int tc = (e->E < m->minE) || e->complete;
   e->complete = tc;
   if (tc) return 0;
   int made = 0;
   if (next == cur) {
      c->t->scatter_events++;
      /* MONSEL_MaterialScatterModel::scatter (:93-134): the cache was set at E_prev by this step */
      if (total != 0.) {
         double rr = cmo_uniform(c->r) * total;
         int index = 0;
         while (cum[index] < rr) index++;
         made = mech_scatter(s, &m->mech[index], e, se, c->r);
      }
      e->complete = (e->E < m->minE) || e->complete;
      if (made) {
         /* MonteCarloSS::trackSecondaryElectron (:165-174) */
         double minE = s->msms[s->regions[se->region].msm].minE;
         if (!(se->E > minE)) made = 0;
      }
      return made;
   }
   else if (next >= 0) {
      c->t->barrier_events++;
      barrier_scatter(s, m, e, next, &hit, 1, c->r);
      double p[3];
      candidate_point(e, SMALL_DISP, p);
      memcpy(e->pos, p, sizeof(p));
      if (!shape_contains(s, s->regions[e->region].shape, e->pos)) e->region = containing_subregion(s, c->chamber, e->pos);
      return 0;
   }
   tally_escape(c, e);
   e->region = -1;
   e->complete = 1;
   return 0;
}

int cmo_run(cmo_scene* s, int chamber, double beam_width, double beam_energy, const double center[3], int nprim,
            uint64_t seed, int nbins, cmo_tally* out)
{
   if (nbins < 1 || nbins > 1024) return -1;
   cmo_rng r;
   cmo_rng_seed(&r, seed);
   run_ctx c = { s, chamber, { 0 }, out, &r };
   memset(out, 0, sizeof(*out));
   /* BackscatterStats(monte, nbins): energy histogram over [0, beam energy in eV] */
   histo_init(&c.h, 0.0, beam_energy * FROMSI_EV, nbins);
   histo_init(&c.h_el, 0.0, PI, 180);
   histo_init(&c.h_az, 0.0, 2.0 * PI, 360);
   electron* stack = (electron*)malloc(sizeof(electron) * STACKMAX);
   for (int i = 0; i < nprim; ++i) {
      /* GaussianBeam::createElectron (GaussianBeam.cu:52-65) + initializeTrajectory (MonteCarloSS.cu:99-105) */
      electron e;
      memset(&e, 0, sizeof(e));
      double rr = sqrt(-2. * log(cmo_uniform(&r))) * beam_width;
      double th = 2.0 * PI * cmo_uniform(&r);
      e.pos[0] = center[0] + rr * cos(th);
      e.pos[1] = center[1] + rr * sin(th);
      e.pos[2] = center[2];
      e.E = e.Eprev = beam_energy;
      e.region = containing_subregion(s, chamber, e.pos);
      int depth = 0;
      electron cur = e;
      for (;;) {
         /* allElectronsComplete (:194-207) */
         while (cur.complete && depth > 0) cur = stack[--depth];
         if (cur.complete) break;
         electron se;
         if (take_step(&c, &cur, &se)) {
            if (depth < STACKMAX) {
               stack[depth++] = cur;
               cur = se;
               out->secondaries++;
            }
         }
      }
      out->trajectories++;
   }
   free(stack);
   return 0;
}

/* ---------------------------------------------------------------- per-function entry points */
void cmo_eval_nistmott_method(cmo_scene* s, int Z, int method, int n, const double* E, const double* u, double* sigma,
                              double* theta, int* ndev)
{
   const mott_elem* m = &s->mott[Z];
   for (int i = 0; i < n; ++i) {
      cmo_rng r = { u + 2 * i, 2, 0, { 0 } };
      sigma[i] = nistmott_sigma(m, E[i], method);
      theta[i] = nistmott_angle(m, E[i], method, &r, s->options & 1);
      ndev[i] = r.used;
   }
}

void cmo_eval_nistmott(cmo_scene* s, int Z, int n, const double* E, const double* u, double* sigma, double* theta,
                       int* ndev)
{
   cmo_eval_nistmott_method(s, Z, 1, n, E, u, sigma, theta, ndev);
}

void cmo_eval_table(cmo_scene* s, int table, int n, const double* x3, int order, double* out)
{
   for (int i = 0; i < n; ++i) out[i] = table_interp(&s->tables[table], x3 + 3 * i, order, s->options & 1);
}

void cmo_eval_tabulated(cmo_scene* s, int msm, int mech, int n, const double* in, double* out)
{
   cmo_eval_tabulated_stride(s, msm, mech, n, in, out, 9);
}

int cmo_table_window(cmo_scene* s, int table, double x0)
{
   int loc[2];
   cmo_nu_locate(x0, s->tables[table].x[0], s->tables[table].n[0], 3, loc);
   return loc[0];
}

void cmo_eval_tabulated_stride(cmo_scene* s, int msm, int mech, int n, const double* in, double* out, int stride)
{
   const mechanism* k = &s->msms[msm].mech[mech];
   for (int i = 0; i < n; ++i) {
      const double* q = in + 9 * i;
      double* o = out + stride * i;
      electron e, se;
      memset(&e, 0, sizeof(e));
      e.E = e.Eprev = q[0];
      e.theta = q[1];
      e.phi = q[2];
      cmo_rng r = { q + 3, 6, 0, { 0 } };
      o[0] = tabulated_rate(s, k, e.E);
      int made = tabulated_scatter(s, k, &e, &se, &r);
      o[1] = e.E;
      o[2] = e.theta;
      o[3] = e.phi;
      o[4] = made;
      o[5] = made ? se.E : 0;
      o[6] = made ? se.theta : 0;
      o[7] = made ? se.phi : 0;
      o[8] = r.used;
      if (stride > 9) o[9] = g_last_theta;
   }
}

void cmo_eval_elastic(cmo_scene* s, int msm, int mech, int n, const double* in, double* out)
{
   const mechanism* k = &s->msms[msm].mech[mech];
   for (int i = 0; i < n; ++i) {
      const double* q = in + 7 * i;
      double* o = out + 5 * i;
      electron e;
      memset(&e, 0, sizeof(e));
      e.E = e.Eprev = q[0];
      e.theta = q[1];
      e.phi = q[2];
      cmo_rng r = { q + 3, 4, 0, { 0 } };
      double cum[MAXEL];
      o[0] = elastic_set_cache(s, k, e.E, cum) * k->densityNa;
      int Z = 0;
      elastic_scatter(s, k, &e, &r, &Z);
      o[1] = e.theta;
      o[2] = e.phi;
      o[3] = Z;
      o[4] = r.used;
   }
}

void cmo_eval_pmma(cmo_scene* s, int msm, int n, const double* in, double* out)
{
   const msm_t* m = &s->msms[msm];
   const mechanism* fitted = NULL;
   const mechanism* polaron = NULL;
   for (int i = 0; i < m->nmech; ++i) {
      if (m->mech[i].kind == M_FITTED) fitted = &m->mech[i];
      if (m->mech[i].kind == M_POLARON) polaron = &m->mech[i];
   }
   for (int i = 0; i < n; ++i) {
      electron e;
      memset(&e, 0, sizeof(e));
      e.E = in[2 * i];
      out[3 * i] = jln_compute(&m->csd, in[2 * i + 1], e.E);
      out[3 * i + 1] = fitted ? mech_rate(s, fitted, &e) : 0;
      out[3 * i + 2] = polaron ? mech_rate(s, polaron, &e) : 0;
   }
}

void cmo_eval_phonon(cmo_scene* s, int msm, int mech, int n, const double* in, double* out)
{
   const mechanism* k = &s->msms[msm].mech[mech];
   for (int i = 0; i < n; ++i) {
      const double* q = in + 5 * i;
      double* o = out + 6 * i;
      electron e;
      memset(&e, 0, sizeof(e));
      e.E = e.Eprev = q[0];
      e.theta = q[1];
      e.phi = q[2];
      cmo_rng r = { q + 3, 2, 0, { 0 } };
      o[0] = phonon_rate(k, e.E);
      phonon_scatter(k, &e, &r);
      o[1] = e.E;
      o[2] = e.theta;
      o[3] = e.phi;
      o[4] = e.Eprev;
      o[5] = r.used;
   }
}

void cmo_eval_shape(cmo_scene* s, int shape, int n, const double* p01, double* out)
{
   for (int i = 0; i < n; ++i) {
      const double* p0 = p01 + 6 * i;
      const double* p1 = p0 + 3;
      nvec v = shape_first_normal(s, shape, p0, p1);
      for (int k = 0; k < 4; ++k) out[6 * i + k] = v.v[k];
      out[6 * i + 4] = shape_contains(s, shape, p0);
      out[6 * i + 5] = shape_contains2(s, shape, p0, p1);
   }
}

void cmo_eval_barrier(cmo_scene* s, int from_region, int to_region, int struck_shape, int n, const double* in,
                      double* out)
{
   (void)struck_shape;
   const msm_t* m = &s->msms[s->regions[from_region].msm];
   for (int i = 0; i < n; ++i) {
      const double* q = in + 6 * i;
      double* o = out + 7 * i;
      electron e;
      memset(&e, 0, sizeof(e));
      e.E = e.Eprev = q[0];
      e.theta = q[1];
      e.phi = q[2];
      memcpy(e.pos, q + 3, 3 * sizeof(double));
      e.region = from_region;
      nvec hit = { { 0., 0., -1., 0.5 } };
      cmo_rng r;
      cmo_rng_seed(&r, 1);
      barrier_scatter(s, m, &e, to_region, &hit, 1, &r);
      o[0] = e.E;
      o[1] = e.theta;
      o[2] = e.phi;
      memcpy(o + 3, e.pos, 3 * sizeof(double));
      o[6] = e.region;
   }
}

void cmo_eval_freepath(cmo_scene* s, int msm, int n, const double* in, double* out)
{
   const msm_t* m = &s->msms[msm];
   for (int i = 0; i < n; ++i) {
      electron e;
      memset(&e, 0, sizeof(e));
      e.E = in[2 * i];
      cmo_rng r = { in + 2 * i + 1, 1, 0, { 0 } };
      double cum[MAXMECH], total;
      out[i] = msm_free_path(s, m, &e, cum, &total, &r);
   }
}

/* MONSEL_MaterialScatterModel::scatter (MONSEL_MaterialScatterModel.cu:93-134): the mechanism the deviate
 * picks from the cumulative rates at E; in[2n] = E u, out[2n] = index (-1: no rate), total rate (1/m) */
void cmo_eval_pick(cmo_scene* s, int msm, int n, const double* in, double* out)
{
   const msm_t* m = &s->msms[msm];
   for (int i = 0; i < n; ++i) {
      electron e;
      memset(&e, 0, sizeof(e));
      e.E = in[2 * i];
      double cum[MAXMECH];
      const double total = msm_set_cache(s, m, &e, cum);
      int index = -1;
      if (total != 0.) {
         const double rr = in[2 * i + 1] * total;
         index = 0;
         while (cum[index] < rr) index++;
      }
      out[2 * i] = index;
      out[2 * i + 1] = total;
   }
}

/* NULagrangeInterpolation::locate (JMONSELutils/NULagrangeInterpolation.cu:5-68) on every axis of a table:
 * out[6n] = (first, nearest) per axis, -1 for axes the table does not have */
void cmo_table_locate(cmo_scene* s, int table, int n, const double* x3, int order, int* out)
{
   const nu_table* t = &s->tables[table];
   for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) {
         int loc[2] = { -1, -1 };
         if (k < t->dim) cmo_nu_locate(x3[3 * i + k], t->x[k], t->n[k], order, loc);
         out[6 * i + 2 * k] = loc[0];
         out[6 * i + 2 * k + 1] = loc[1];
      }
}

void cmo_eval_beam(int n, const double* in, double* out)
{
   for (int i = 0; i < n; ++i) {
      const double* q = in + 6 * i;
      double rr = sqrt(-2. * log(q[4])) * q[0];
      double th = 2.0 * PI * q[5];
      out[3 * i] = q[1] + rr * cos(th);
      out[3 * i + 1] = q[2] + rr * sin(th);
      out[3 * i + 2] = q[3];
   }
}
