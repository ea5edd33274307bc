// cm_device.cuh -- per-event device arithmetic of the transport path.
//
// Templated on the compute precision R (double for the plain form, float for
// the batched form); positions and the plane solves are double in both.
// Units: eV, nm, 1/nm.  Each function cites the reference source it follows
// (paths relative to CudaMONSEL/CudaMONSEL/gov/nist/).
#pragma once
#include <math.h>
#include <stdint.h>

#include "cm_scene.h"

namespace cm {

#define CM_HD __host__ __device__ __forceinline__
// every per-event function is host-callable as well, so the same code can be
// exercised on the CPU by test harnesses
#define CM_D __host__ __device__ __forceinline__

CM_D uint32_t umulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

CM_D int popcount64(unsigned long long x) {
#ifdef __CUDA_ARCH__
  return __popcll(x);
#else
  return __builtin_popcountll(x);
#endif
}

// ------------------------------------------------------------ counter-based RNG
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), keyed per electron.
struct U4 { uint32_t x, y, z, w; };

CM_D U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = umulhi32(M0, c0), lo0 = M0 * c0;
    uint32_t hi1 = umulhi32(M1, c2), lo1 = M1 * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += W0; k1 += W1;
  }
  return {c0, c1, c2, c3};
}

CM_HD uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// Deviate source for one event: counter (step, sub) of the electron's stream.
// Uniforms lie in the open interval (0, 1).
template <typename R> struct Rng;

template <> struct Rng<double> {
  uint32_t k0, k1, step, sub;
  U4 buf;
  int left;
  CM_D Rng(uint64_t key, uint32_t st, uint32_t sb) : k0((uint32_t)key), k1((uint32_t)(key >> 32)), step(st), sub(sb), left(0) {}
  CM_D double next() {
    if (left == 0) { buf = philox(step, sub++, 0x5eedu, 0u, k0, k1); left = 2; }
    uint32_t a, b;
    if (left == 2) { a = buf.x; b = buf.y; } else { a = buf.z; b = buf.w; }
    --left;
    uint64_t x = (((uint64_t)a << 32) | b) >> 11;
    return ((double)x + 0.5) * (1.0 / 9007199254740992.0);
  }
};

template <> struct Rng<float> {
  uint32_t k0, k1, step, sub;
  U4 buf;
  int left;
  CM_D Rng(uint64_t key, uint32_t st, uint32_t sb) : k0((uint32_t)key), k1((uint32_t)(key >> 32)), step(st), sub(sb), left(0) {}
  CM_D float next() {
    if (left == 0) { buf = philox(step, sub++, 0x5eedu, 0u, k0, k1); left = 4; }
    uint32_t a = left == 4 ? buf.x : left == 3 ? buf.y : left == 2 ? buf.z : buf.w;
    --left;
    return ((float)(a >> 8) + 0.5f) * (1.0f / 16777216.0f);
  }
};

// A fixed list of deviates (the per-function parity entry points inject the oracle's)
template <typename R> struct FixedRng {
  const double* u;
  int n, used;
  CM_D R next() { R v = used < n ? (R)u[used] : R(0.5); ++used; return v; }
};

// ------------------------------------------------------------ precision helpers
template <typename R> CM_D R msqrt(R x);
template <> CM_D double msqrt(double x) { return sqrt(x); }
template <> CM_D float msqrt(float x) { return sqrtf(x); }
template <typename R> CM_D R mlog(R x);
template <> CM_D double mlog(double x) { return log(x); }
template <> CM_D float mlog(float x) { return logf(x); }
template <typename R> CM_D R mexp(R x);
template <> CM_D double mexp(double x) { return exp(x); }
template <> CM_D float mexp(float x) { return expf(x); }
template <typename R> CM_D R mpow(R x, R y);
template <> CM_D double mpow(double x, double y) { return pow(x, y); }
template <> CM_D float mpow(float x, float y) { return powf(x, y); }
template <typename R> CM_D R macos(R x);
template <> CM_D double macos(double x) { return acos(x); }
template <> CM_D float macos(float x) { return acosf(x); }
template <typename R> CM_D R matan2(R y, R x);
template <> CM_D double matan2(double y, double x) { return atan2(y, x); }
template <> CM_D float matan2(float y, float x) { return atan2f(y, x); }
template <typename R> CM_D void msincos(R x, R* s, R* c);
template <> CM_D void msincos(double x, double* s, double* c) { sincos(x, s, c); }
template <> CM_D void msincos(float x, float* s, float* c) { sincosf(x, s, c); }
template <typename R> CM_D R mcos(R x);
template <> CM_D double mcos(double x) { return cos(x); }
template <> CM_D float mcos(float x) { return cosf(x); }
template <typename R> CM_D R mround(R x);
template <> CM_D double mround(double x) { return round(x); }
template <> CM_D float mround(float x) { return roundf(x); }
template <typename R> CM_D R msinh(R x);
template <> CM_D double msinh(double x) { return sinh(x); }
template <> CM_D float msinh(float x) { return sinhf(x); }

// acos(1 - 2 q^2) with the reference's clamps (NISTMottRS.cu:148-149):
// com > -1 ? (com < 1 ? acos(com) : 0) : pi.  In float the equivalent
// 2 asin(|q|) keeps full relative precision for small angles.
template <typename R> CM_D R angle_from_q(R q);
template <> CM_D double angle_from_q(double q) {
  const double com = 1.0 - (2.0 * q * q);
  return com > -1.0 ? (com < 1.0 ? acos(com) : 0.0) : kPi;
}
template <> CM_D float angle_from_q(float q) {
  const float a = fabsf(q);
  if (a >= 1.0f) return (float)kPi;
  return 2.0f * asinf(a);
}

// acos(1 - t) for t >= 0; float uses 2 asin(sqrt(t / 2)), which keeps its
// relative precision for the small angles of screened Rutherford scattering
template <typename R> CM_D R acos_1m(R t);
template <> CM_D double acos_1m(double t) { return acos(1.0 - t); }
template <> CM_D float acos_1m(float t) { return 2.0f * asinf(sqrtf(fminf(fmaxf(0.5f * t, 0.0f), 1.0f))); }

// acos(1 - 2 r) for r in (0, 1) (isotropic polar angle); float uses 2 asin(sqrt(r))
template <typename R> CM_D R iso_angle(R r);
template <> CM_D double iso_angle(double r) { return acos(1 - 2.0 * r); }
template <> CM_D float iso_angle(float r) { return 2.0f * asinf(sqrtf(r)); }

// select by value (no address of a local array is taken: keeps the values in registers)
template <typename R> CM_D R sel4(R a0, R a1, R a2, R a3, int k) { return k <= 0 ? a0 : k == 1 ? a1 : k == 2 ? a2 : a3; }

// ------------------------------------------------------------ uniform-grid Lagrange
// JMONSELutils/ULagrangeInterpolation.cu:5-33, order 3, written out with
// scalars: Neville's tableau on f0..f3 at reduced x, starting from the nearest
// node and walking the correction path the reference walks.
template <typename R> CM_D R uneville3(R f0, R f1, R f2, R f3, R x) {
  int ns = (int)mround(x);
  if (ns < 0) ns = 0;
  else if (ns > 3) ns = 3;
  R c0 = f0, c1 = f1, c2 = f2, c3 = f3;
  R d0 = f0, d1 = f1, d2 = f2;
  R y = sel4(c0, c1, c2, c3, ns);
  --ns;
  R dy, w;
  // m = 1
  w = c1 - d0; d0 = -((R)1 - x) * w / (R)1; c0 = -((R)0 - x) * w / (R)1;
  w = c2 - d1; d1 = -((R)2 - x) * w / (R)1; c1 = -((R)1 - x) * w / (R)1;
  w = c3 - d2; d2 = -((R)3 - x) * w / (R)1; c2 = -((R)2 - x) * w / (R)1;
  if (2 * ns < 1) dy = sel4(c0, c1, c2, c3, ns + 1);
  else { dy = sel4(d0, d1, d2, d2, ns); --ns; }
  y += dy;
  // m = 2
  w = c1 - d0; d0 = -((R)2 - x) * w / (R)2; c0 = -((R)0 - x) * w / (R)2;
  w = c2 - d1; d1 = -((R)3 - x) * w / (R)2; c1 = -((R)1 - x) * w / (R)2;
  if (2 * ns < 0) dy = sel4(c0, c1, c2, c2, ns + 1);
  else { dy = sel4(d0, d1, d1, d1, ns); --ns; }
  y += dy;
  // m = 3
  w = c1 - d0; d0 = -((R)3 - x) * w / (R)3; c0 = -((R)0 - x) * w / (R)3;
  if (2 * ns < -1) dy = c0;
  else dy = d0;
  y += dy;
  return y;
}

// ULagrangeInterpolation.cu:35-48
// The grid coordinate, the window index and the offset inside the window are
// computed in double in both precisions: a float coordinate of up to 60 grid
// steps keeps only ~1e-5 of a step, which the cubic turns into ~1e-6 relative
// error; the table values and the Neville recursion stay in R.
template <typename T, typename R> CM_D T ulagrange_d1_as(const R* f, int len, double x0, double xinc, double x) {
  const double reducedx = (x - x0) / xinc;
  int index0 = (int)reducedx - 1;
  if (index0 < 0) index0 = 0;
  else if (index0 > len - 4) index0 = len - 4;
  return uneville3((T)f[index0], (T)f[index0 + 1], (T)f[index0 + 2], (T)f[index0 + 3], (T)(reducedx - (double)index0));
}

template <typename R> CM_D R ulagrange_d1(const R* f, int len, double x0, double xinc, double x) {
  return ulagrange_d1_as<R, R>(f, len, x0, xinc, x);
}

// ULagrangeInterpolation.cu:80-103, f row-major [n0][n1]
template <typename R>
CM_D R ulagrange_d2(const R* f, int n0, int n1, double x00, double x01, double xinc0, double xinc1, double xa,
                    double xb) {
  const double reducedx1 = (xa - x00) / xinc0;
  int index0 = (int)reducedx1 - 1;
  if (index0 < 0) index0 = 0;
  else if (index0 > n0 - 4) index0 = n0 - 4;
  // the recursion runs in double (the NISTMott quantile table is read from its double copy in both
  // precisions): neighbouring quantiles cancel in the cubic, which cost float up to ~2e-6 of the angle
  double y[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) y[i] = ulagrange_d1_as<double>(f + (size_t)(index0 + i) * n1, n1, x01, xinc1, xb);
  // the final 1-D step runs on the 4 values with x0 moved to the window start
  const double x0w = x00 + (double)index0 * xinc0;
  const double reducedx = (xa - x0w) / xinc0;
  return (R)uneville3(y[0], y[1], y[2], y[3], reducedx);
}

// ------------------------------------------------------------ non-uniform Lagrange
// JMONSELutils/NULagrangeInterpolation.cu:5-68
template <typename R> CM_D void nu_locate(R x, const R* xs, int n, int order, int& first, int& nearest) {
  int lowlim = -1, uplim = n, maxindex = n - 1;
  bool ascending = xs[maxindex] > xs[0];
  while ((uplim - lowlim) > 1) {
    int mid = (uplim + lowlim) >> 1;
    if ((x > xs[mid]) == ascending) lowlim = mid;
    else uplim = mid;
  }
  if (lowlim < 0) { first = 0; nearest = 0; return; }
  if (uplim > maxindex) { first = maxindex - order; nearest = maxindex; return; }
  const R xl = xs[lowlim], xu = xs[uplim];
  if (ascending) nearest = ((x - xl) <= (xu - x)) ? lowlim : uplim;
  else nearest = ((xl - x) <= (x - xu)) ? lowlim : uplim;
  int firstInd = lowlim, lastInd = uplim;
  while (((lastInd - firstInd) < order) && (firstInd > 0) && (lastInd < maxindex)) {
    if (((((xl - xs[firstInd - 1]) + xu) - xs[lastInd + 1]) >= 0) == ascending) lastInd += 1;
    else firstInd -= 1;
  }
  if (lastInd >= maxindex) first = maxindex - order;
  else if (firstInd <= 0) first = 0;
  else first = firstInd;
}

// NULagrangeInterpolation.cu:85-112 with order 3: Neville on (xv[i], fv[i]),
// i = 0..3, from the nearest node ns, written out with scalars
template <typename R> CM_D R nu_neville3(const R* fv, const R* xv, int ns, R x) {
  const R x0 = xv[0], x1 = xv[1], x2 = xv[2], x3 = xv[3];
  R c0 = fv[0], c1 = fv[1], c2 = fv[2], c3 = fv[3];
  R d0 = c0, d1 = c1, d2 = c2;
  R y = sel4(c0, c1, c2, c3, ns);
  --ns;
  R dy, w, ho, hp, den;
  // m = 1
  ho = x0 - x; hp = x1 - x; w = c1 - d0; den = w / (ho - hp); d0 = hp * den; c0 = ho * den;
  ho = x1 - x; hp = x2 - x; w = c2 - d1; den = w / (ho - hp); d1 = hp * den; c1 = ho * den;
  ho = x2 - x; hp = x3 - x; w = c3 - d2; den = w / (ho - hp); d2 = hp * den; c2 = ho * den;
  if ((2 * ns) < 1) dy = sel4(c0, c1, c2, c3, ns + 1);
  else { dy = sel4(d0, d1, d2, d2, ns); --ns; }
  y += dy;
  // m = 2
  ho = x0 - x; hp = x2 - x; w = c1 - d0; den = w / (ho - hp); d0 = hp * den; c0 = ho * den;
  ho = x1 - x; hp = x3 - x; w = c2 - d1; den = w / (ho - hp); d1 = hp * den; c1 = ho * den;
  if ((2 * ns) < 0) dy = sel4(c0, c1, c2, c2, ns + 1);
  else { dy = sel4(d0, d1, d1, d1, ns); --ns; }
  y += dy;
  // m = 3
  ho = x0 - x; hp = x3 - x; w = c1 - d0; den = w / (ho - hp); d0 = hp * den; c0 = ho * den;
  if ((2 * ns) < -1) dy = c0;
  else dy = d0;
  y += dy;
  return y;
}

// order-1 Neville (linear), NULagrangeInterpolation.cu:85-112 with order 1:
// y starts at the nearest node and takes one correction (c[0] when the
// nearest node is the first, d[0] otherwise).
template <typename R> CM_D R nu_neville1(R f0, R f1, R x0, R x1, int ns, R x) {
  const R ho = x0 - x, hp = x1 - x;
  const R den = (f1 - f0) / (ho - hp);
  return ns == 0 ? f0 + ho * den : f1 + hp * den;
}

// Window selection of every table lookup: NULagrangeInterpolation::locate on the axis's double copy with
// the argument promoted to double, so FP32 picks exactly the window and nearest node the reference picks
// for the same (float) argument; comparing with float-rounded abscissae would move the boundaries.
CM_D void nu_window(double x, const double* xsd, int n, int order, int& first, int& nearest) {
  nu_locate<double>(x, xsd, n, order, first, nearest);
}

// NULagrangeInterpolation.cu:131-147 for a 1-D table, order 1 (TabulatedInelasticSM::scatterRate)
template <typename R> CM_D R nu_d1_order1(const R* f, const R* xs, const double* xsd, int n, R x) {
  int first, nearest;
  nu_window((double)x, xsd, n, 1, first, nearest);
  return nu_neville1(f[first], f[first + 1], xs[first], xs[first + 1], nearest - first, x);
}

// Lagrange weights of the cubic through the 4 abscissae xv at x.  d2 and d3 evaluate many cubics on
// the same abscissae at the same point (every row of a window), so the weights are formed once and
// each row is a 4-term dot product instead of a Neville tableau; the value is the same polynomial.
template <typename R> CM_D void lag4(const R* xv, R x, R w[4]) {
  const R d0 = x - xv[0], d1 = x - xv[1], d2 = x - xv[2], d3 = x - xv[3];
  w[0] = (d1 * d2 * d3) / ((xv[0] - xv[1]) * (xv[0] - xv[2]) * (xv[0] - xv[3]));
  w[1] = (d0 * d2 * d3) / ((xv[1] - xv[0]) * (xv[1] - xv[2]) * (xv[1] - xv[3]));
  w[2] = (d0 * d1 * d3) / ((xv[2] - xv[0]) * (xv[2] - xv[1]) * (xv[2] - xv[3]));
  w[3] = (d0 * d1 * d2) / ((xv[3] - xv[0]) * (xv[3] - xv[1]) * (xv[3] - xv[2]));
}

template <typename R> CM_D R dot4(const R w[4], const R* f) { return w[0] * f[0] + w[1] * f[1] + w[2] * f[2] + w[3] * f[3]; }

// NULagrangeInterpolation.cu:169-192 on a 2-D table (order 3)
template <typename R>
CM_D R nu_d2(const R* f, const R* xs0, const double* xs0d, int n0, const R* xs1, const double* xs1d, int n1, R xa, R xb) {
  int i0, near0;
  nu_window((double)xa, xs0d, n0, 3, i0, near0);
  int j0, near1;
  nu_window((double)xb, xs1d, n1, 3, j0, near1);
  R xv1[4] = {xs1[j0], xs1[j0 + 1], xs1[j0 + 2], xs1[j0 + 3]};
  R w1[4];
  lag4(xv1, xb, w1);
  R y[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) y[i] = dot4(w1, f + (size_t)(i0 + i) * n1 + j0);
  R xv0[4] = {xs0[i0], xs0[i0 + 1], xs0[i0 + 2], xs0[i0 + 3]};
  R w0[4];
  lag4(xv0, xa, w0);
  return dot4(w0, y);
}

// NULagrangeInterpolation.cu:215-240 on a 3-D table (order 3).  The reference's
// final 1-D step uses xsamp[0][0..3] (line 236) whatever the window; `fixes`
// uses the window's own abscissae.  Evaluated in double in both precisions (see Table).
CM_D double nu_d3(const double* f, const double* xs0, int n0, const double* xs1, int n1, const double* xs2, int n2,
                  double xa, double xb, double xc, bool fixes) {
  using R = double;
  int i0, near0, j0, near1, k0, near2;
  nu_window((double)xa, xs0, n0, 3, i0, near0);
  nu_window((double)xb, xs1, n1, 3, j0, near1);
  nu_window((double)xc, xs2, n2, 3, k0, near2);
  R xv1[4] = {xs1[j0], xs1[j0 + 1], xs1[j0 + 2], xs1[j0 + 3]};
  R xv2[4] = {xs2[k0], xs2[k0 + 1], xs2[k0 + 2], xs2[k0 + 3]};
  R w1[4], w2[4];
  lag4(xv1, xb, w1);
  lag4(xv2, xc, w2);
  R y[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    R z[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) z[j] = dot4(w2, f + ((size_t)(i0 + i) * n1 + (j0 + j)) * n2 + k0);
    y[i] = dot4(w1, z);
  }
  const int base = fixes ? i0 : 0;
  R xv0[4] = {xs0[base], xs0[base + 1], xs0[base + 2], xs0[base + 3]};
  R w0[4];
  lag4(xv0, xa, w0);
  return dot4(w0, y);
}

// the staged prefix of the table blob (kernels launched with it hold s.nstaged elements here)
extern __shared__ __align__(16) unsigned char cm_stage_smem[];

// an array of the table blob: from shared memory when the kernel staged it, else from global memory
template <typename R> CM_D const R* blob_at(const SceneView<R>& s, int off) {
#ifdef __CUDA_ARCH__
  if (off < s.nstaged) return reinterpret_cast<const R*>(cm_stage_smem) + off;
#endif
  return s.blob + off;
}

// NUTableInterpolation::interpolate (JMONSEL/NUTableInterpolation.cu:98-115)
template <typename R> CM_D R table_interp(const SceneView<R>& s, int t, R x0, R x1, R x2, int order) {
  const Table& tb = s.tables[t];
  const R* v = blob_at(s, tb.off_v);
  if (tb.dim == 1) {
    const double* xsd = s.dbl + tb.off_x64[0];
    if (order == 1) return nu_d1_order1(v, blob_at(s, tb.off_x[0]), xsd, tb.n[0], x0);
    int first, nearest;
    const R* xs = blob_at(s, tb.off_x[0]);
    nu_window((double)x0, xsd, tb.n[0], 3, first, nearest);
    R fv[4] = {v[first], v[first + 1], v[first + 2], v[first + 3]};
    R xv[4] = {xs[first], xs[first + 1], xs[first + 2], xs[first + 3]};
    return nu_neville3(fv, xv, nearest - first, x0);
  }
  if (tb.dim == 2)
    return nu_d2(v, blob_at(s, tb.off_x[0]), s.dbl + tb.off_x64[0], tb.n[0], blob_at(s, tb.off_x[1]),
                 s.dbl + tb.off_x64[1], tb.n[1], x0, x1);
  return (R)nu_d3(s.dbl + tb.off_v64, s.dbl + tb.off_x64[0], tb.n[0], s.dbl + tb.off_x64[1], tb.n[1],
                          s.dbl + tb.off_x64[2], tb.n[2], (double)x0, (double)x1, (double)x2, (s.options & 1) != 0);
}

// The windows NUTableInterpolation::interpolate selects for (x0, x1, x2): (first, nearest) per axis,
// order 1 on a 1-D table as scatterRate uses it, else 3; unused axes give -1.
template <typename R> CM_D void table_windows(const SceneView<R>& s, int t, R x0, R x1, R x2, int order, int out[6]) {
  const Table& tb = s.tables[t];
  const R xs[3] = {x0, x1, x2};
  for (int k = 0; k < 3; ++k) {
    out[2 * k] = out[2 * k + 1] = -1;
    if (k < tb.dim) nu_window((double)xs[k], s.dbl + tb.off_x64[k], tb.n[k], tb.dim == 1 ? order : 3, out[2 * k],
                              out[2 * k + 1]);
  }
}

// ------------------------------------------------------------ elastic scattering
// EPQLibrary/BrowningEmpiricalCrossSection.cu:24-29, sigma in m^2, E in eV
template <typename R> CM_D R browning_sigma(const Mott& m, R E) {
  const R e = E / R(1000);
  const R re = msqrt(e);
  const R z17 = (R)m.zp17;
  return R(3.0e-22) * z17 / (e + R(0.005) * z17 * re + R(0.0007) * (R)m.zp2 / re);
}

// BrowningEmpiricalCrossSection.cu:31-45.  The reference reads z through a
// reference bound to a temporary Element (BrowningEmpiricalCrossSection.cuh:20,
// instances built from ints at BrowningEmpiricalCrossSection.cu:47-...); the
// compiled reference reads 0, so r/(r+1) is NaN and every angle is isotropic.
// `fixes` uses the element's atomic number.
template <typename R, typename G> CM_D R browning_angle(const Mott& m, R E, G& g, bool fixes) {
  const R r1 = g.next(), r2 = g.next();
  if (!fixes) return iso_angle(r2);
  const R z = (R)m.Z;
  const R e = E / R(1000);
  const R r = (R(300.0) * e / z) + ((R)m.zp3 / (R(3.0e5) * e));
  if (r1 <= r / (r + 1)) {
    const R alpha = R(7.0e-3) / e;
    return acos_1m((R(2.0) * alpha * r2) / (alpha - r2 + 1));
  }
  return iso_angle(r2);
}

// JMONSEL/NISTMottRS.cu:103-119 times the SelectableElasticSM rate factor (1/nm); below the
// extrapolation energy method 3 is linear in E, methods 1 and 2 scale Browning's cross section
template <typename R> CM_D R nistmott_rate(const SceneView<R>& s, const Mott& m, int method, R kel, R kbrown, R E, R logE) {
  if (E < (R)m.extrapolateBelowEnergy[method]) {
    if (method == 3) return kel * (R)m.mottXSatMin[3] * E / (R)m.extrapolateBelowEnergy[3];
    return (R)m.sfBrowning[method] * browning_sigma(m, E) * kbrown;
  }
  if (E < (R)s.maxMott) {
    return kel * ulagrange_d1(blob_at(s, m.off_spwem), 61, s.dl50, s.param, (double)logE);
  }
  // ScreenedRutherfordScatteringAngle.cu:24-30
  return (R)m.rutherfordA / (E + (R)m.rutherfordB) * kbrown;
}

// NISTMottRS.cu:121-154 (Browning's angles below the extrapolation energy for every method)
template <typename R, typename G> CM_D R nistmott_angle(const SceneView<R>& s, const Mott& m, int method, R E, G& g) {
  if (E < (R)m.extrapolateBelowEnergy[method]) return browning_angle(m, E, g, (s.options & 1) != 0);
  if (E < (R)s.maxMott) {
    const double lg = log((double)E);  // double in both precisions: see ulagrange_d1
    const R u = g.next();
    const double q = ulagrange_d2(s.dbl + m.off_x1d, 61, 201, s.dl50, 0.0, s.param, 0.005, lg, (double)u);
    if (sizeof(R) == 4) {  // theta near pi: asin is ill-conditioned near 1, so q is not rounded to float first
      const double a = fabs(q);
      return a >= 1.0 ? (R)kPi : (R)(2.0 * asin(a));
    }
    return angle_from_q((R)q);
  }
  // ScreenedRutherfordScatteringAngle.cu:32-39; in double in both precisions (1 + alpha - r cancels for
  // deviates near 1)
  const double alpha = m.rutherfordAlpha / (double)E;
  const double r = (double)g.next();
  return (R)acos_1m(2.0 * alpha * r / (1 + alpha - r));
}

// ------------------------------------------------------------ direction algebra
// Electron::updateDirection (NISTMonte/Electron.cu:111-131) on a unit vector.
// When the direction is exactly along z the reference's phi is 0 for every
// electron that reaches here with sin(theta) == 0, so cp = 1, sp = 0.
template <typename R> CM_D void update_dir(R d[3], R dTheta, R dPhi) {
  const R ct = d[2];
  const R st = msqrt(d[0] * d[0] + d[1] * d[1]);
  R cp = 1, sp = 0;
  if (st > 0) { cp = d[0] / st; sp = d[1] / st; }
  R sa, ca, sb, cb;
  msincos(dTheta, &sa, &ca);
  msincos(dPhi, &sb, &cb);
  const R xx = (cb * ct * sa) + (ca * st);
  const R yy = sa * sb;
  const R dx = (cp * xx) - (sp * yy);
  const R dy = (cp * yy) + (sp * xx);
  const R dz = (ca * ct) - (cb * sa * st);
  const R inv = R(1) / msqrt(dx * dx + dy * dy + dz * dz);
  d[0] = dx * inv; d[1] = dy * inv; d[2] = dz * inv;
}

template <typename R> CM_D void dir_from_angles(R d[3], R theta, R phi) {
  R st, ct, sp, cp;
  msincos(theta, &st, &ct);
  msincos(phi, &sp, &cp);
  d[0] = st * cp; d[1] = st * sp; d[2] = ct;
}

// kE / (1 + x)^(2/3) - kE, the Nieminen loss of JoyLuoNieminenCSD.cu:104.  In
// float the difference of two nearly equal numbers loses everything for
// short steps; kE * expm1(-2/3 log1p(x)) is the same quantity without the
// cancellation.
template <typename R> CM_D R nieminen_loss(R kE, R x);
template <> CM_D double nieminen_loss(double kE, double x) { return (kE / pow(1. + x, 2. / 3.)) - kE; }
template <> CM_D float nieminen_loss(float kE, float x) { return kE * expm1f(-(2.0f / 3.0f) * log1pf(x)); }

// ------------------------------------------------------------ slowing down
// JMONSEL/JoyLuoNieminenCSD.cu:91-121; the recursive halving is run with an
// explicit stack in the same order (first half, then second half at the
// energy reached after the first).
template <typename R> CM_D R jln_compute(const Jln& c, R len, R kE) {
  if ((c.nce == 0) || (kE < (R)c.minE) || (kE <= R(0))) return 0;
  if (kE <= (R)c.breakE) return nieminen_loss(kE, R(1.5) * (R)c.gamma * len * kE * msqrt(kE));
  // The reference halves the step recursively while the loss exceeds 10 % of
  // the energy (JoyLuoNieminenCSD.cu:101-121).  The segments form a binary tree
  // visited depth first, left half first; node (depth, idx) covers
  // len / 2^depth.  Walking it with the index alone needs no stack: after a
  // leaf, climb while idx is a right child, then step to the right sibling.
  // Halves still pending = depth - popcount(idx), bounded like a 46-deep stack.
  R total = 0;
  int depth = 0;
  unsigned long long idx = 0;
  for (;;) {
    R l = len;
    for (int k = 0; k < depth; ++k) l = l / 2;
    const R e = kE + total;
    bool leaf = true;
    if ((e < (R)c.minE) || (e <= R(0))) {
    } else if (e <= (R)c.breakE) {
      total += nieminen_loss(e, R(1.5) * (R)c.gamma * l * e * msqrt(e));
    } else {
      R loss = 0;
      for (int i = 0; i < c.nce; i++) loss += (R)c.coef[i] * mlog(((R)c.recipJ[i] * e) + (R)c.beta[i]);
      loss *= l / e;
      const int pending = depth - popcount64(idx);
      if (loss <= (R(0.1) * e) || pending >= 46 || depth >= 62) total += -loss;
      else leaf = false;
    }
    if (!leaf) {  // descend into the first half
      ++depth;
      idx <<= 1;
      continue;
    }
    while (depth > 0 && (idx & 1ULL)) {
      idx >>= 1;
      --depth;
    }
    if (depth == 0) break;
    idx |= 1ULL;  // the second half of the same parent
  }
  return total;
}

// ------------------------------------------------------------ mechanism rates
// TabulatedInelasticSM.cu:436-459
template <typename R> CM_D R tabulated_rate(const SceneView<R>& s, const Mech& k, R E) {
  const R kEa = E + (R)k.energyOffset;
  if (kEa < (R)k.iimfpDomain0) return 0;
  return (R)k.rateMult * table_interp(s, k.tIIMFP, kEa, R(0), R(0), 1);
}

// GanachaudMokraniPhononInelasticSM.cu:46-72
template <typename R> CM_D R phonon_rate(const Mech& k, R kE) {
  // GanachaudMokraniPhononInelasticSM::scatterRate (GanachaudMokraniPhononInelasticSM.cu:46-72).  The energy
  // ratio and the branch decisions are taken in double in both precisions (kE is exact in either), so a
  // float phonon energy never moves an energy near threshold to the other branch; the common small-x
  // form then runs in the compute precision, the rare x >= 0.1 form (E < 10 hbar omega) in double.
  if ((double)kE < k.phononE) return 0;
  const double xd = k.phononE / (double)kE;
  if (xd < 0.1) {
    const R x = (R)xd;
    return (R)k.prefactor * x * mlog(R(4) / x);
  }
  if (xd >= 1.0) return 0;
  const double t = sqrt(1.0 - xd);
  return (R)(k.prefactor * xd * log((1.0 + t) / (1.0 - t)));
}

// ------------------------------------------------------------ geometry (double)
struct NV { double n[3]; double u; };

CM_D NV nv_none() { NV r; r.n[0] = r.n[1] = r.n[2] = 0.; r.u = INFINITY; return r; }

// NormalMultiPlaneShape.cu:26-38
CM_D bool tie_break(const double* n) {
  if (n[0] < 0.) return false;
  if (n[0] == 0.) {
    if (n[1] < 0.) return false;
    if (n[1] == 0.)
      if (n[2] < 0.) return false;
  }
  return true;
}

// NormalMultiPlaneShape.cu:40-171
CM_D NV planes_first_normal(const Plane* pl, int np, const double* p0, const double* p1) {
  double umin = -INFINITY, umax = INFINITY;
  int minindex = -1, maxindex = -1;
  const double delta[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
  for (int i = 0; i < np; i++) {
    const Plane& P = pl[i];
    const double pmc[3] = {p0[0] - P.p[0], p0[1] - P.p[1], p0[2] - P.p[2]};
    const double num = (pmc[0] * P.n[0]) + (pmc[1] * P.n[1]) + (pmc[2] * P.n[2]);
    const double den = (delta[0] * P.n[0]) + (delta[1] * P.n[1]) + (delta[2] * P.n[2]);
    if (den == 0) {
      if ((num < 0) || ((num == 0) && tie_break(P.n))) continue;
      return nv_none();
    }
    const double u = -num / den;
    if (den > 0) {
      if (u < umax) {
        if ((u < 0) || (u <= umin)) return nv_none();
        umax = u;
        maxindex = i;
      }
    } else if (u > umin) {
      if ((u > 1) || (u >= umax)) return nv_none();
      umin = u;
      minindex = i;
    }
  }
  NV r;
  if (umin > 0) {
    r.u = umin;
    r.n[0] = pl[minindex].n[0]; r.n[1] = pl[minindex].n[1]; r.n[2] = pl[minindex].n[2];
    return r;
  }
  if ((umax <= 1) && (umax > 0.)) {
    r.u = umax;
    r.n[0] = pl[maxindex].n[0]; r.n[1] = pl[maxindex].n[1]; r.n[2] = pl[maxindex].n[2];
    return r;
  }
  return nv_none();
}

// MultiPlaneShape.cu:23-27 (Plane::contains)
CM_D bool plane_contains(const Plane& P, const double* p) {
  return (((p[0] - P.p[0]) * P.n[0] + (p[1] - P.p[1]) * P.n[1] + (p[2] - P.p[2]) * P.n[2]) <= 0.0);
}

// NormalMultiPlaneShape.cu:178-204.  The reference writes delta[0] three times
// and leaves delta[1], delta[2] unset; they are 0 here.
CM_D bool planes_contains2(const Plane* pl, int np, const double* p0, const double* p1) {
  bool didDelta = false;
  double delta[3] = {0., 0., 0.};
  for (int i = 0; i < np; i++) {
    const Plane& P = pl[i];
    const double p0c[3] = {p0[0] - P.p[0], p0[1] - P.p[1], p0[2] - P.p[2]};
    const double dn = (p0c[0] * P.n[0]) + (p0c[1] * P.n[1]) + (p0c[2] * P.n[2]);
    if (dn > 0.) return false;
    if (dn == 0.) {
      if (!didDelta) {
        delta[0] = p1[2] - p0[2];
        didDelta = true;
      }
      const double dd = (delta[0] * P.n[0]) + (delta[1] * P.n[1]) + (delta[2] * P.n[2]);
      if (dd > 0.) return false;
      if ((dd == 0.) && !tie_break(P.n)) return false;
    }
  }
  return true;
}

// Sphere.cu:11-14
CM_D bool sphere_contains(const Shape& sh, const double* p) {
  const double a = p[0] - sh.c[0], b = p[1] - sh.c[1], c = p[2] - sh.c[2];
  return a * a + b * b + c * c <= sh.r * sh.r;
}

// Sphere.cu:21-45
CM_D double sphere_first_intersection(const Shape& sh, const double* p0, const double* p1) {
  const double d[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
  const double m[3] = {p0[0] - sh.c[0], p0[1] - sh.c[1], p0[2] - sh.c[2]};
  const double ma2 = -2.0 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double b = 2.0 * (m[0] * d[0] + m[1] * d[1] + m[2] * d[2]);
  const double c2 = 2.0 * ((m[0] * m[0] + m[1] * m[1] + m[2] * m[2]) - sh.r * sh.r);
  const double f = b * b + ma2 * c2;
  if (f >= 0) {
    const double sf = sqrt(f);
    double up = (b + sf) / ma2, un = (b - sf) / ma2;
    if (up < 0.0) up = INFINITY;
    if (un < 0.0) un = INFINITY;
    return fmin(up, un);
  }
  return INFINITY;
}

// CylindricalShape::contains (NISTMonte/CylindricalShape.cu:31-48)
CM_D bool cylinder_contains(const Shape& sh, const double* p) {
  const double u = (sh.ax[0] * (p[0] - sh.e0[0]) + sh.ax[1] * (p[1] - sh.e0[1]) + sh.ax[2] * (p[2] - sh.e0[2])) / sh.len2;
  const double a = p[0] - (sh.e0[0] + u * sh.ax[0]), b = p[1] - (sh.e0[1] + u * sh.ax[1]),
               c = p[2] - (sh.e0[2] + u * sh.ax[2]);
  return (u >= 0) && (u <= 1.0) && ((a * a + b * b + c * c) <= sh.rad2);
}

// NormalCylindricalShape::contains(pos0, pos1) (NormalCylindricalShape.cu:24-98)
CM_D bool cylinder_contains2(const Shape& sh, const double* pos0, const double* pos1) {
  const double* na = sh.nax;
  const double p0c[3] = {pos0[0] - sh.e0[0], pos0[1] - sh.e0[1], pos0[2] - sh.e0[2]};
  const double p0cdotn = (p0c[0] * na[0]) + (p0c[1] * na[1]) + (p0c[2] * na[2]);
  const double p0cSquared = (p0c[0] * p0c[0]) + (p0c[1] * p0c[1]) + (p0c[2] * p0c[2]);
  const double r2 = p0cSquared - (p0cdotn * p0cdotn);
  const bool on_end0 = (p0cdotn == 0) && (r2 <= sh.rad2);
  const bool on_end1 = (p0cdotn == sh.len) && (r2 <= sh.rad2);
  const bool on_cylinder = (r2 == sh.rad2) && (p0cdotn >= 0) && (p0cdotn <= sh.len);
  const double delta[3] = {pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2]};
  if (on_end0 || on_end1) {
    const double dd = (delta[0] * na[0]) + (delta[1] * na[1]) + (delta[2] * na[2]);
    if (dd == 0) {
      if (na[0] == 0) return na[1] == 0 ? na[2] > 0 : na[1] > 0;
      return na[0] > 0;
    }
    return on_end0 ? dd > 0 : dd < 0;
  }
  if (on_cylinder) {
    const double nv[3] = {p0c[0] - (p0cdotn * na[0]), p0c[1] - (p0cdotn * na[1]), p0c[2] - (p0cdotn * na[2])};
    return ((nv[0] * delta[0]) + (nv[1] * delta[1]) + (nv[2] * delta[2])) < 0;
  }
  return (r2 < sh.rad2) && (p0cdotn > 0) && (p0cdotn < sh.len);
}

// NormalCylindricalShape::getFirstNormal (NormalCylindricalShape.cu:111-322): the end caps,
// then the wall's quadratic; the first crossing in (0, 1] with its outward normal
CM_D NV cylinder_first_normal(const Shape& sh, const double* pos0, const double* pos1) {
  NV nv = nv_none();
  const double* na = sh.nax;
  const double radius2 = sh.rad2, mLen = sh.len, mLen2 = sh.len2;
  const double p0c[3] = {pos0[0] - sh.e0[0], pos0[1] - sh.e0[1], pos0[2] - sh.e0[2]};
  const double p0cSquared = (p0c[0] * p0c[0]) + (p0c[1] * p0c[1]) + (p0c[2] * p0c[2]);
  const double delta[3] = {pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2]};
  const double p0cdotn = (p0c[0] * na[0]) + (p0c[1] * na[1]) + (p0c[2] * na[2]);
  const double deltadotn = (delta[0] * na[0]) + (delta[1] * na[1]) + (delta[2] * na[2]);
  const double deltadotnSquared = deltadotn * deltadotn;
  const double p0cdotdelta = (delta[0] * p0c[0]) + (delta[1] * p0c[1]) + (delta[2] * p0c[2]);
  const double deltaSquared = (delta[0] * delta[0]) + (delta[1] * delta[1]) + (delta[2] * delta[2]);
  int which = 0;
  double u1 = 0., u2 = 0., saved = 0.;
  if (deltadotn != 0.) {
    u1 = -p0cdotn / deltadotn;
    if ((u1 > 0.) && (u1 <= 1.) && ((p0cSquared + (2 * u1 * p0cdotdelta) + (u1 * u1 * deltaSquared)) <= radius2)) {
      nv.u = u1;
      which = 1;
    }
    u2 = u1 + (mLen / deltadotn);
    if ((u2 > 0.) && (u2 <= 1.) && (u2 < nv.u) &&
        (((p0cSquared + (2 * u2 * p0cdotdelta) + (u2 * u2 * deltaSquared) + mLen2) -
          (2 * mLen * (p0cdotn + (u2 * deltadotn)))) <= radius2)) {
      nv.u = u2;
      which = 2;
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
        for (int root = 0; root < 2; ++root) {
          const double u = (minusbover2 + (root == 0 ? term : -term)) / a;
          if ((u > 0) && (u <= 1) && (u < nv.u)) {
            const double projection = p0cdotn + (u * deltadotn);
            if ((projection >= 0) && (projection <= mLen)) {
              nv.u = u;
              which = 3;
              saved = projection;
            }
          }
        }
      }
    }
  }
  if (which == 1 || which == 2) {
    const double sg = which == 1 ? -1.0 : 1.0;
    nv.n[0] = sg * na[0];
    nv.n[1] = sg * na[1];
    nv.n[2] = sg * na[2];
  } else if (which == 3) {
    const double v[3] = {(p0c[0] + (nv.u * delta[0])) - (saved * na[0]), (p0c[1] + (nv.u * delta[1])) - (saved * na[1]),
                         (p0c[2] + (nv.u * delta[2])) - (saved * na[2])};
    const double mag = sqrt((v[0] * v[0]) + (v[1] * v[1]) + (v[2] * v[2]));
    nv.n[0] = v[0] / mag;
    nv.n[1] = v[1] / mag;
    nv.n[2] = v[2] / mag;
  }
  return nv;
}

// out-of-line copies for the shape-tree walks, which would otherwise inline the
// cylinder at every level of the tree (the leaf-only kernels inline it)
__host__ __device__ __noinline__ bool cylinder_contains2_call(const Shape& sh, const double* pos0, const double* pos1) {
  return cylinder_contains2(sh, pos0, pos1);
}
__host__ __device__ __noinline__ NV cylinder_first_normal_call(const Shape& sh, const double* pos0, const double* pos1) {
  return cylinder_first_normal(sh, pos0, pos1);
}

// a leaf shape (plane set, sphere or cylinder) holds p
template <typename R> CM_D bool leaf_contains(const SceneView<R>& s, const Shape& sh, const double* p) {
  if (sh.kind == SHAPE_PLANES) {
    for (int i = 0; i < sh.np; ++i)
      if (!plane_contains(s.planes[sh.plane0 + i], p)) return false;
    return true;
  }
  if (sh.kind == SHAPE_CYLINDER) return cylinder_contains(sh, p);
  return sphere_contains(sh, p);
}

template <typename R, bool INL = true>
CM_D bool leaf_contains2(const SceneView<R>& s, const Shape& sh, const double* p0, const double* p1) {
  if (sh.kind == SHAPE_PLANES) return planes_contains2(s.planes + sh.plane0, sh.np, p0, p1);
  if (sh.kind == SHAPE_CYLINDER) return INL ? cylinder_contains2(sh, p0, p1) : cylinder_contains2_call(sh, p0, p1);
  return sphere_contains(sh, p0);
}

// D bounds the intersection/union nesting of the scene's shapes; D = 0: leaf
// shapes only (intersections of plane sets merged into one plane set when the
// scene was built), so no tree walk is compiled in.
// NormalIntersectionShape::contains = A && B, NormalUnionShape (SumShape) = A || B.
template <typename R, int D> struct Contains {
  static __host__ __device__ __noinline__ bool eval(const SceneView<R>& s, int id, const double* p) {
    const Shape& sh = s.shapes[id];
    if (sh.kind == SHAPE_INTERSECTION)
      return Contains<R, D - 1>::eval(s, sh.a, p) && Contains<R, D - 1>::eval(s, sh.b, p);
    if (sh.kind == SHAPE_UNION) return Contains<R, D - 1>::eval(s, sh.a, p) || Contains<R, D - 1>::eval(s, sh.b, p);
    return leaf_contains(s, sh, p);
  }
  static __host__ __device__ __noinline__ bool eval2(const SceneView<R>& s, int id, const double* p0, const double* p1) {
    const Shape& sh = s.shapes[id];
    if (sh.kind == SHAPE_INTERSECTION)
      return Contains<R, D - 1>::eval2(s, sh.a, p0, p1) && Contains<R, D - 1>::eval2(s, sh.b, p0, p1);
    if (sh.kind == SHAPE_UNION)
      return Contains<R, D - 1>::eval2(s, sh.a, p0, p1) || Contains<R, D - 1>::eval2(s, sh.b, p0, p1);
    return leaf_contains2<R, false>(s, sh, p0, p1);
  }
};

template <typename R> struct Contains<R, 0> {
  static CM_D bool eval(const SceneView<R>& s, int id, const double* p) { return leaf_contains(s, s.shapes[id], p); }
  static CM_D bool eval2(const SceneView<R>& s, int id, const double* p0, const double* p1) {
    return leaf_contains2<R, false>(s, s.shapes[id], p0, p1);
  }
};

// Leaves are tested inline; a tree of intersections only is the AND of its
// leaves, walked with a small stack; trees holding a union recurse out of line.
template <typename R, int D = kMaxShapeDepth> CM_D bool shape_contains(const SceneView<R>& s, int id, const double* p) {
  const Shape& top = s.shapes[id];
  if (D == 0 || (top.kind != SHAPE_INTERSECTION && top.kind != SHAPE_UNION)) return leaf_contains(s, top, p);
  if (top.anyunion) return Contains<R, D>::eval(s, id, p);
  int stack[D + 2];
  int sp = 0;
  stack[sp++] = id;
  while (sp > 0) {
    const Shape& sh = s.shapes[stack[--sp]];
    if (sh.kind == SHAPE_INTERSECTION) {
      if (sp + 2 > D + 2) return Contains<R, D>::eval(s, id, p);
      stack[sp++] = sh.b;
      stack[sp++] = sh.a;
    } else if (!leaf_contains(s, sh, p)) {
      return false;
    }
  }
  return true;
}

// NormalShape::contains(p0, p1) inside the tree walks (cylinders out of line)
template <typename R, int D> CM_D bool tree_contains2(const SceneView<R>& s, int id, const double* p0, const double* p1) {
  const Shape& top = s.shapes[id];
  if (D == 0 || (top.kind != SHAPE_INTERSECTION && top.kind != SHAPE_UNION)) return leaf_contains2<R, false>(s, top, p0, p1);
  if (top.anyunion) return Contains<R, D>::eval2(s, id, p0, p1);
  int stack[D + 2];
  int sp = 0;
  stack[sp++] = id;
  while (sp > 0) {
    const Shape& sh = s.shapes[stack[--sp]];
    if (sh.kind == SHAPE_INTERSECTION) {
      if (sp + 2 > D + 2) return Contains<R, D>::eval2(s, id, p0, p1);
      stack[sp++] = sh.b;
      stack[sp++] = sh.a;
    } else if (!leaf_contains2<R, false>(s, sh, p0, p1)) {
      return false;
    }
  }
  return true;
}

template <typename R, int D = kMaxShapeDepth>
CM_D bool shape_contains2(const SceneView<R>& s, int id, const double* p0, const double* p1) {
  if (D == 0) return leaf_contains2<R, true>(s, s.shapes[id], p0, p1);
  return tree_contains2<R, D>(s, id, p0, p1);
}

template <typename R, int D> struct FirstNormal;

// NormalIntersectionShape.cu:19-239
template <typename R, int D> __host__ __device__ __noinline__ NV inter_first_normal(const SceneView<R>& s, const Shape& sh, const double* pos0,
                                                                           const double* pos1) {
  const NV none = nv_none();
  int adepth, bdepth;
  double u;
  const double delta[3] = {pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2]};
  NV nva = FirstNormal<R, D - 1>::eval(s, sh.a, pos0, pos1);
  if (nva.u <= 1.) adepth = ((delta[0] * nva.n[0]) + (delta[1] * nva.n[1]) + (delta[2] * nva.n[2])) > 0 ? 1 : 0;
  else {
    if (!tree_contains2<R, D - 1>(s, sh.a, pos0, pos1)) return none;
    adepth = 1;
  }
  NV nvb = FirstNormal<R, D - 1>::eval(s, sh.b, pos0, pos1);
  if (nvb.u <= 1.) bdepth = ((delta[0] * nvb.n[0]) + (delta[1] * nvb.n[1]) + (delta[2] * nvb.n[2])) > 0 ? 1 : 0;
  else {
    if (!tree_contains2<R, D - 1>(s, sh.b, pos0, pos1)) return none;
    if (adepth == 1) return nva;
    bdepth = 1;
  }
  int cdepth = adepth + bdepth;
  const double EXTRAU = 1.e-10;
  for (int guard = 0; guard < 4096; ++guard) {
    if (nva.u < nvb.u) {
      if (bdepth == 1) return nva;
      cdepth ^= 1;
      u = nva.u + EXTRAU;
      const double tmp[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
      nva = FirstNormal<R, D - 1>::eval(s, sh.a, tmp, pos1);
      if (nva.u < INFINITY) nva.u = (nva.u * (1. - u)) + u;
      if (nva.u > 1) return cdepth == 0 ? none : nvb;
      adepth ^= 1;
    } else if (nva.u > nvb.u) {
      if (adepth == 1) return nvb;
      cdepth ^= 1;
      u = nvb.u + EXTRAU;
      const double tmp[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
      nvb = FirstNormal<R, D - 1>::eval(s, sh.b, tmp, pos1);
      if (nvb.u < INFINITY) nvb.u = (nvb.u * (1. - u)) + u;
      if (nvb.u > 1) return cdepth == 0 ? none : nva;
      bdepth ^= 1;
    } else {
      const int depthchange = (((adepth ^ 1) - adepth) + (bdepth ^ 1)) - bdepth;
      if (depthchange == 0) {
        u = nva.u + EXTRAU;
        const double t1[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
        nva = FirstNormal<R, D - 1>::eval(s, sh.a, t1, pos1);
        if (nva.u < INFINITY) nva.u = (nva.u * (1. - u)) + u;
        u = nvb.u + EXTRAU;
        const double t2[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
        nvb = FirstNormal<R, D - 1>::eval(s, sh.b, t2, pos1);
        if (nvb.u < INFINITY) nvb.u = (nvb.u * (1. - u)) + u;
        if (nva.u > 1) return adepth == 0 ? nvb : none;
        if (nvb.u > 1) return bdepth == 0 ? nva : none;
        adepth ^= 1;
        bdepth ^= 1;
      } else {
        NV r;
        r.n[0] = (nva.n[0] + nvb.n[0]) / 2.;
        r.n[1] = (nva.n[1] + nvb.n[1]) / 2.;
        r.n[2] = (nva.n[2] + nvb.n[2]) / 2.;
        r.u = nva.u;
        return r;
      }
    }
  }
  return none;
}

// NormalUnionShape.cu:40-269: the crossings of A and B in order along the step,
// tracking the depth (number of shapes the point is inside); a crossing where the
// union's depth changes to or from 0 is the union's boundary
template <typename R, int D> __host__ __device__ __noinline__ NV union_first_normal(const SceneView<R>& s, const Shape& sh,
                                                                           const double* pos0, const double* pos1) {
  const NV none = nv_none();
  int adepth, bdepth;
  double u;
  const double delta[3] = {pos1[0] - pos0[0], pos1[1] - pos0[1], pos1[2] - pos0[2]};
  NV nva = FirstNormal<R, D - 1>::eval(s, sh.a, pos0, pos1);
  if (nva.u <= 1.) adepth = ((delta[0] * nva.n[0]) + (delta[1] * nva.n[1]) + (delta[2] * nva.n[2])) > 0 ? 1 : 0;
  else {
    if (tree_contains2<R, D - 1>(s, sh.a, pos0, pos1)) return none;
    adepth = 0;
  }
  NV nvb = FirstNormal<R, D - 1>::eval(s, sh.b, pos0, pos1);
  if (nvb.u <= 1.) bdepth = ((delta[0] * nvb.n[0]) + (delta[1] * nvb.n[1]) + (delta[2] * nvb.n[2])) > 0 ? 1 : 0;
  else {
    if (tree_contains2<R, D - 1>(s, sh.b, pos0, pos1)) return none;
    return nva;
  }
  int cdepth = adepth + bdepth;
  const double EXTRAU = 1.e-10;
  for (int guard = 0; guard < 4096; ++guard) {
    if (nva.u < nvb.u) {
      if (adepth == cdepth) return nva;
      cdepth = cdepth == 1 ? 2 : 1;
      u = nva.u + EXTRAU;
      const double tmp[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
      nva = FirstNormal<R, D - 1>::eval(s, sh.a, tmp, pos1);
      if (nva.u < INFINITY) nva.u = (nva.u * (1. - u)) + u;
      if (nva.u > 1) return cdepth == bdepth ? nvb : none;
      adepth ^= 1;
    } else if (nva.u > nvb.u) {
      if (bdepth == cdepth) return nvb;
      cdepth = cdepth == 1 ? 2 : 1;
      u = nvb.u + EXTRAU;
      const double tmp[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
      nvb = FirstNormal<R, D - 1>::eval(s, sh.b, tmp, pos1);
      if (nvb.u < INFINITY) nvb.u = (nvb.u * (1. - u)) + u;
      if (nvb.u > 1) return cdepth == adepth ? nva : none;
      bdepth ^= 1;
    } else {
      const int depthchange = (((adepth ^ 1) - adepth) + (bdepth ^ 1)) - bdepth;
      if (depthchange == 0) {
        u = nva.u + EXTRAU;
        const double t1[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
        nva = FirstNormal<R, D - 1>::eval(s, sh.a, t1, pos1);
        if (nva.u < INFINITY) nva.u = (nva.u * (1. - u)) + u;
        u = nvb.u + EXTRAU;
        const double t2[3] = {pos0[0] + (u * delta[0]), pos0[1] + (u * delta[1]), pos0[2] + (u * delta[2])};
        nvb = FirstNormal<R, D - 1>::eval(s, sh.b, t2, pos1);
        if (nvb.u < INFINITY) nvb.u = (nvb.u * (1. - u)) + u;
        if (nva.u > 1) return cdepth != bdepth ? nvb : none;
        if (nvb.u > 1) return cdepth != adepth ? nva : none;
        adepth ^= 1;
        bdepth ^= 1;
      } else {
        NV r;
        r.n[0] = (nva.n[0] + nvb.n[0]) / 2.;
        r.n[1] = (nva.n[1] + nvb.n[1]) / 2.;
        r.n[2] = (nva.n[2] + nvb.n[2]) / 2.;
        r.u = nva.u;
        return r;
      }
    }
  }
  return none;
}

template <typename R, bool INL = true>
CM_D NV leaf_first_normal(const SceneView<R>& s, const Shape& sh, const double* p0, const double* p1) {
  if (sh.kind == SHAPE_PLANES) return planes_first_normal(s.planes + sh.plane0, sh.np, p0, p1);
  if (sh.kind == SHAPE_CYLINDER) return INL ? cylinder_first_normal(sh, p0, p1) : cylinder_first_normal_call(sh, p0, p1);
  NV r = nv_none();
  if (sh.kind == SHAPE_SPHERE) r.u = sphere_first_intersection(sh, p0, p1);
  return r;
}

template <typename R, int D> struct FirstNormal {
  static CM_D NV eval(const SceneView<R>& s, int id, const double* p0, const double* p1) {
    const Shape& sh = s.shapes[id];
    if (sh.kind == SHAPE_INTERSECTION) return inter_first_normal<R, D>(s, sh, p0, p1);
    if (sh.kind == SHAPE_UNION) return union_first_normal<R, D>(s, sh, p0, p1);
    return leaf_first_normal<R, false>(s, sh, p0, p1);
  }
};

template <typename R> struct FirstNormal<R, 0> {
  static CM_D NV eval(const SceneView<R>& s, int id, const double* p0, const double* p1) {
    return leaf_first_normal<R, false>(s, s.shapes[id], p0, p1);
  }
};

template <typename R, int D = kMaxShapeDepth>
CM_D NV shape_first_normal(const SceneView<R>& s, int id, const double* p0, const double* p1) {
  if (D == 0) return leaf_first_normal<R, true>(s, s.shapes[id], p0, p1);
  return FirstNormal<R, D>::eval(s, id, p0, p1);
}

// Region boxes (built on the host, padded against rounding) let a step skip the
// children it cannot reach; the children that remain are tested in the same
// order as before, so the region found and its tie-breaks are unchanged.
CM_D bool point_in_box(const double* bb, const double* p) {
  return p[0] >= bb[0] && p[1] >= bb[1] && p[2] >= bb[2] && p[0] <= bb[3] && p[1] <= bb[4] && p[2] <= bb[5];
}

// the segment p0 -> p1 meets the box (slab test over u in [0, 1])
CM_D bool segment_meets_box(const double* bb, const double* p0, const double* p1) {
  double lo = 0.0, hi = 1.0;
  for (int a = 0; a < 3; ++a) {
    const double d = p1[a] - p0[a];
    if (d == 0.0) {
      if (p0[a] < bb[a] || p0[a] > bb[3 + a]) return false;
      continue;
    }
    double t0 = (bb[a] - p0[a]) / d, t1 = (bb[3 + a] - p0[a]) / d;
    if (t0 > t1) {
      const double t = t0;
      t0 = t1;
      t1 = t;
    }
    lo = t0 > lo ? t0 : lo;
    hi = t1 < hi ? t1 : hi;
    if (lo > hi) return false;
  }
  return true;
}

// RegionBase.cu:50-60, iterative: the first child whose shape holds p owns it
// the first child of r (in list order) whose shape holds p, or -1
template <typename R, int D> CM_D int first_child_holding(const SceneView<R>& s, const Region& r, const double* p) {
  if (r.grid < 0) {
    for (int i = 0; i < r.nchild; ++i) {
      const int c = s.children[r.child0 + i];
      if (point_in_box(s.regions[c].bb, p) && shape_contains<R, D>(s, s.regions[c].shape, p)) return c;
    }
    return -1;
  }
  // the cell's children and the unbounded ones, merged in list order
  const ChildGrid& g = s.grids[r.grid];
  int a = 0, na = 0;
  const double fx = floor((p[0] - g.x0) / g.dx), fy = floor((p[1] - g.y0) / g.dy);
  if (fx >= 0.0 && fy >= 0.0 && fx < (double)g.nx && fy < (double)g.ny) {
    const int cell = g.cell0 + (int)fy * g.nx + (int)fx;
    a = s.cell_start[cell];
    na = s.cell_start[cell + 1] - a;
  }
  const int b = g.unb0, nb = g.nunb;
  int ia = 0, ib = 0;
  while (ia < na || ib < nb) {
    int pos;
    if (ib >= nb || (ia < na && s.grid_items[a + ia] < s.grid_items[b + ib])) pos = s.grid_items[a + ia++];
    else pos = s.grid_items[b + ib++];
    const int c = s.children[r.child0 + pos];
    if (point_in_box(s.regions[c].bb, p) && shape_contains<R, D>(s, s.regions[c].shape, p)) return c;
  }
  return -1;
}

template <typename R, int D = kMaxShapeDepth> CM_D int containing_subregion(const SceneView<R>& s, int reg, const double* p) {
  if (!shape_contains<R, D>(s, s.regions[reg].shape, p)) return -1;
  for (int depth = 0; depth < 64; ++depth) {
    const int found = first_child_holding<R, D>(s, s.regions[reg], p);
    if (found < 0) return reg;
    reg = found;
  }
  return reg;
}

template <typename R> CM_D bool is_containing_region(const SceneView<R>& s, int reg, int target) {
  // target lies below reg iff walking up from target reaches reg
  int t = s.regions[target].parent;
  for (int depth = 0; depth < 64 && t >= 0; ++depth) {
    if (t == reg) return true;
    t = s.regions[t].parent;
  }
  return false;
}

// RegionBase.cu:74-119.  p1 is clipped to the boundary; returns the region just
// over it (-1: outside the chamber) and the struck boundary's normal.
template <typename R, int D = kMaxShapeDepth>
CM_D int find_end_of_step(const SceneView<R>& s, int reg, const double* p0, double* p1, double* hitn,
                          bool* clipped = nullptr) {
  const Region& r = s.regions[reg];
  int base = reg;
  NV nv = shape_first_normal<R, D>(s, r.shape, p0, p1);
  double t = nv.u;
  hitn[0] = nv.n[0]; hitn[1] = nv.n[1]; hitn[2] = nv.n[2];
  if ((t <= 1.0) && r.parent >= 0) base = r.parent;
  if (r.grid < 0) {
    for (int i = 0; i < r.nchild; ++i) {
      const int c = s.children[r.child0 + i];
      if (!segment_meets_box(s.regions[c].bb, p0, p1)) continue;
      NV cn = shape_first_normal<R, D>(s, s.regions[c].shape, p0, p1);
      if ((cn.u <= 1.0) && (cn.u < t)) {
        t = cn.u;
        base = c;
        hitn[0] = cn.n[0]; hitn[1] = cn.n[1]; hitn[2] = cn.n[2];
      }
    }
  } else {
    // the in-order scan keeps the first child of smallest u below the region's own crossing:
    // here children come cell by cell, so ties go to the lower list position explicitly
    int bpos = 0x7fffffff;
    auto visit = [&](int pos) {
      const int c = s.children[r.child0 + pos];
      if (!segment_meets_box(s.regions[c].bb, p0, p1)) return;
      NV cn = shape_first_normal<R, D>(s, s.regions[c].shape, p0, p1);
      if ((cn.u <= 1.0) && ((cn.u < t) || (cn.u == t && bpos != 0x7fffffff && pos < bpos))) {
        t = cn.u;
        base = c;
        bpos = pos;
        hitn[0] = cn.n[0]; hitn[1] = cn.n[1]; hitn[2] = cn.n[2];
      }
    };
    const ChildGrid& g = s.grids[r.grid];
    for (int k = 0; k < g.nunb; ++k) visit(s.grid_items[g.unb0 + k]);
    // cells crossed by the step's x-y projection, in order along the step, until past the best crossing
    const double ex = p1[0] - p0[0], ey = p1[1] - p0[1];
    const double X1 = g.x0 + g.nx * g.dx, Y1 = g.y0 + g.ny * g.dy;
    double tlo = 0.0, thi = 1.0;
    bool hit = true;
    if (ex == 0.0) hit = p0[0] >= g.x0 && p0[0] <= X1;
    else {
      double a0 = (g.x0 - p0[0]) / ex, a1 = (X1 - p0[0]) / ex;
      if (a0 > a1) { const double q = a0; a0 = a1; a1 = q; }
      tlo = a0 > tlo ? a0 : tlo;
      thi = a1 < thi ? a1 : thi;
    }
    if (ey == 0.0) hit = hit && p0[1] >= g.y0 && p0[1] <= Y1;
    else {
      double a0 = (g.y0 - p0[1]) / ey, a1 = (Y1 - p0[1]) / ey;
      if (a0 > a1) { const double q = a0; a0 = a1; a1 = q; }
      tlo = a0 > tlo ? a0 : tlo;
      thi = a1 < thi ? a1 : thi;
    }
    if (hit && tlo <= thi) {
      int ix = (int)floor((p0[0] + tlo * ex - g.x0) / g.dx), iy = (int)floor((p0[1] + tlo * ey - g.y0) / g.dy);
      ix = ix < 0 ? 0 : (ix >= g.nx ? g.nx - 1 : ix);
      iy = iy < 0 ? 0 : (iy >= g.ny ? g.ny - 1 : iy);
      const int sx = ex > 0.0 ? 1 : (ex < 0.0 ? -1 : 0), sy = ey > 0.0 ? 1 : (ey < 0.0 ? -1 : 0);
      double tx = sx == 0 ? INFINITY : ((g.x0 + (ix + (sx > 0 ? 1 : 0)) * g.dx) - p0[0]) / ex;
      double ty = sy == 0 ? INFINITY : ((g.y0 + (iy + (sy > 0 ? 1 : 0)) * g.dy) - p0[1]) / ey;
      const double dtx = sx == 0 ? INFINITY : g.dx / fabs(ex), dty = sy == 0 ? INFINITY : g.dy / fabs(ey);
      double tentry = tlo;
      for (int guard = 0; guard < g.nx + g.ny + 2; ++guard) {
        if (tentry > thi || (t <= 1.0 && tentry > t)) break;
        const int cell = g.cell0 + iy * g.nx + ix;
        for (int k = s.cell_start[cell]; k < s.cell_start[cell + 1]; ++k) visit(s.grid_items[k]);
        if (tx < ty) {
          ix += sx;
          tentry = tx;
          tx += dtx;
        } else {
          iy += sy;
          tentry = ty;
          ty += dty;
        }
        if (ix < 0 || iy < 0 || ix >= g.nx || iy >= g.ny) break;
      }
    }
  }
  if (clipped) *clipped = t <= 1.0;
  if (t <= 1.0) {
    const double delta[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    p1[0] = p0[0] + (t * delta[0]);
    p1[1] = p0[1] + (t * delta[1]);
    p1[2] = p0[2] + (t * delta[2]);
    const double mag = sqrt(delta[0] * delta[0] + delta[1] * delta[1] + delta[2] * delta[2]);
    const double over[3] = {p1[0] + kSmallDispNm * (delta[0] / mag), p1[1] + kSmallDispNm * (delta[1] / mag),
                            p1[2] + kSmallDispNm * (delta[2] / mag)};
    for (int depth = 0; depth < 64 && base >= 0; ++depth) {
      const int res = containing_subregion<R, D>(s, base, over);
      if (res >= 0) return res;
      base = s.regions[base].parent;
    }
    return -1;
  }
  return reg;
}

}  // namespace cm
