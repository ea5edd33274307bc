// cm_scene.h -- flattened scene description shared by host and device.
//
// The host facade records the reference's object graph (Region tree,
// NormalShapes, MONSEL_MaterialScatterModel with its ScatterMechanisms) and
// flattens it into these plain arrays.  Device units: energy in eV, length in
// nm, rates in 1/nm.  Geometry is double precision in every mode.
#pragma once
#include <stdint.h>

namespace cm {

constexpr int kMaxMech = 8;
constexpr int kMaxElem = 8;
constexpr int kMaxCore = 16;
constexpr int kMaxShapeDepth = 4;
constexpr int kGridMinChildren = 24;  // regions with at least this many bounded children get a ChildGrid

// NISTMonte/MonteCarloSS.cu:32-33 in nm
constexpr double kChamberRadiusNm = 0.1e9;
constexpr double kSmallDispNm = 1.0e-6;
constexpr double kPi = 3.14159265358979323846;

enum ShapeKind : int { SHAPE_SPHERE = 1, SHAPE_PLANES = 2, SHAPE_INTERSECTION = 3, SHAPE_CYLINDER = 4, SHAPE_UNION = 5 };
enum MechKind : int { MECH_NISTMOTT = 1, MECH_TABULATED = 2, MECH_FITTED = 3, MECH_PHONON = 4, MECH_POLARON = 5 };

struct Shape {
  int kind;
  int anyunion;      // a union below (or at) this node
  int a, b;          // intersection / union children
  int plane0, np;    // planes [plane0, plane0+np)
  double c[3], r;    // sphere (nm)
  // NormalCylindricalShape (nm): end0, axis = end1 - end0, axis / |axis| as the
  // reference computed it, radius^2, |axis|^2, |axis|
  double e0[3], ax[3], nax[3], rad2, len2, len;
};

struct Plane {
  double n[3];
  double p[3];       // nm
};

struct Region {
  int parent, msm, shape;
  int child0, nchild;  // children indices in Scene::children
  int cls;             // wave segment of electrons in this region (by material model)
  double bb[6];        // axis-aligned box holding the region's shape (nm): min xyz, max xyz
  int grid;            // index of the grid over this region's children, -1: scan them in order
};

// A uniform x-y grid over the children of a region with many of them.  Each cell lists, ascending,
// the positions (in the region's child list) of the children whose box overlaps it; children whose
// box is unbounded in x or y are listed once apart.  Searches visit only the listed children and
// resolve ties by position, so they find what the in-order scan finds.
struct ChildGrid {
  double x0, y0, dx, dy;  // nm
  int nx, ny;
  int cell0;              // cell (ix, iy) lists grid_items[cell_start[cell0 + iy * nx + ix] .. next)
  int unb0, nunb;         // the unbounded children: grid_items[unb0 .. unb0 + nunb)
};

// electrons are kept in one wave segment per material class, so that the
// threads of a warp mostly run the same material's code
constexpr int kClasses = 4;
// a wave has two segments per class: electrons at or above kSegmentSplitEv and below it (the low band
// takes the Browning branch of the elastic cross sections and the low-energy secondary paths), so that
// a warp's threads mostly run the same branches
constexpr int kSegments = 2 * kClasses;
constexpr double kSegmentSplitEv = 50.0;
constexpr int kMaxWave = 1 << 27;  // electrons per wave segment: kSegments x and 8 x (the pool) stay within int

// JoyLuoNieminenCSD (JMONSEL/JoyLuoNieminenCSD.cu:42-121) in eV/nm units
struct Jln {
  int nce;
  double coef[kMaxElem];     // eV^2 / nm
  double recipJ[kMaxElem];   // 1/eV
  double beta[kMaxElem];
  double breakE, gamma, minE;  // eV, eV^-1.5 nm^-1, eV
};

struct Mech {
  int kind;
  // NISTMott via SelectableElasticSM: per element mott index and rate factor
  int nel;
  int mott[kMaxElem];        // index into Scene::mott
  int mottMethod;            // NISTMottRS method 1..3
  double kel[kMaxElem];      // a0^2 * scalefactor * density * N_A in nm^-1 per (table unit)
  double kbrown[kMaxElem];   // the same factor for a Browning/Rutherford cross section in nm^2
  // TabulatedInelasticSM (JMONSEL/TabulatedInelasticSM.cu:461-498), energies in eV
  int methodSE;
  int tIIMFP, tRed, tTheta, tSEE0;
  double energyOffset, minEgenSE, rateMult, energyCBbottom, bandgap, energyGap, offsetFermiEnergy, bEref;
  double eiDomain0, eiDomain1, iimfpDomain0, rangeSE0lo, rangeSE0hi;
  int ncore;
  double core[kMaxCore];
  // FittedInelSM
  double energySEgen, eFermi;
  Jln csd;
  // phonon / polaron
  double phononE, prefactor, extinction, cutoff;
};

struct Msm {
  int material;
  int vacuum;
  int nmech, mech0;          // mechanisms [mech0, mech0+nmech)
  int csd;                   // 0 = ZeroCSD, 1 = JoyLuoNieminenCSD
  Jln jln;
  double minE;               // eV (may be -inf)
  double ecb;                // E_CB bottom of this material, eV
  double u0;                 // barrier's u0 (= E_CB of the material it was built for), eV
  int classical;
  double lambda, lambdaFactor;  // lambdaFactor in 1/sqrt(eV)
};

// NISTMottRS per element; the tables live in the precision blob, the extrapolation constants are
// indexed by method (1: Factory, 2: Factory100, 3: Factory100Lin; entry 0 copies method 1)
struct Mott {
  int Z;
  int off_spwem, off_x1;     // offsets of the cross sections in the table blob (off_x1 unused: -1)
  int off_x1d;               // offset of the 61 x 201 quantile table in the double copies (dbl)
  double extrapolateBelowEnergy[4];  // eV
  double sfBrowning[4];
  double mottXSatMin[4];             // table value (units of a0^2) at extrapolateBelowEnergy
  double zp17, zp2, zp3;
  double rutherfordA, rutherfordB;  // sigma = A / (E + B) in nm^2 with E in eV
  double rutherfordAlpha;           // alpha = rutherfordAlpha / E
};

// NUTableInterpolation (dims 1..3) in the precision blob, with double copies in SceneView::dbl of every
// axis (window selection compares the argument with the reference's abscissae in double in both
// precisions) and of a 3-D table's values (its reference d3 step extrapolates from the first energy
// window, which amplifies rounding by orders of magnitude, so FP32 evaluates it in double too)
struct Table {
  int dim;
  int n[3];
  int off_x[3];
  int off_v;
  int off_x64[3];            // axes in dbl
  int off_v64;               // values in dbl (3-D tables), else -1
  double domain[3][2];
  double range[2];
};

// The whole scene as device pointers (one struct passed by value to kernels)
template <typename R>
struct SceneView {
  const Shape* shapes;
  const Plane* planes;
  const Region* regions;
  const int* children;
  const Msm* msms;
  const Mech* mechs;
  const Mott* mott;
  const Table* tables;
  const ChildGrid* grids;
  const int* cell_start;
  const int* grid_items;
  const R* blob;             // table data in compute precision
  const double* dbl;         // double copies: NISTMott quantile tables (sampled angles within 1e-6 in FP32
                             // too), NU-table axes and 3-D table values
  int chamber;
  int options;               // bit 0: JMONSEL fixes, bit 1: exact CSG in FP32
  int depth;                 // deepest intersection nesting; 0 = every shape is a leaf (plane set or sphere)
  double dl50, param;        // NISTMott log-energy grid (eV)
  double maxMott;            // NISTMottRS MAX_NISTMOTT in eV
  int nstaged;               // elements of blob's prefix this kernel holds in shared memory (0: none)
  int nstage;                // elements of the prefix the scene places for staging (a multiple of 16 bytes)
};

}  // namespace cm
