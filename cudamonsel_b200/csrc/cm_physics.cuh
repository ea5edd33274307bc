// cm_physics.cuh -- the ScatterMechanism / BarrierScatterMechanism events,
// shared by the wavefront kernels and the per-function entry points.
// Units eV / nm; reference paths relative to CudaMONSEL/CudaMONSEL/gov/nist/.
#pragma once
#include "cm_device.cuh"

namespace cm {

// MONSEL_MaterialScatterModel::setCache term for one mechanism (1/nm).
// logE is log(E) (only the NIST Mott grid uses it).
template <typename R> CM_D R mech_rate(const SceneView<R>& s, const Mech& k, R E, R logE) {
  switch (k.kind) {
    case MECH_NISTMOTT: {  // SelectableElasticSM.cu:25-47
      R total = 0;
      for (int i = 0; i < k.nel; ++i) total += nistmott_rate(s, s.mott[k.mott[i]], k.mottMethod, (R)k.kel[i], (R)k.kbrown[i], E, logE);
      return total;
    }
    case MECH_TABULATED:
      return tabulated_rate(s, k, E);
    case MECH_FITTED:  // FittedInelSM.cu:20-25 (a 0.1 nm step's loss, per nm, per SE energy)
      if (E <= (R)(k.energySEgen + k.eFermi)) return 0;
      return (-jln_compute(k.csd, R(0.1), E) * R(10)) / (R)k.energySEgen;
    case MECH_PHONON:
      return phonon_rate(k, E);
    case MECH_POLARON:  // GanachaudMokraniPolaronTrapSM.cu:21-27
      if (E > (R)k.cutoff) return 0;
      return (R)k.prefactor * mexp(-(R)k.extinction * E);
  }
  return 0;
}

// TabulatedInelasticSM::updateDirection on angles (TabulatedInelasticSM.cu:68-85)
template <typename R> CM_D void update_angles(R& theta, R& phi, R dTheta, R dPhi) {
  R st, ct, sp, cp, sa, ca, sb, cb;
  msincos(theta, &st, &ct);
  msincos(phi, &sp, &cp);
  msincos(dTheta, &sa, &ca);
  msincos(dPhi, &sb, &cb);
  const R xx = (cb * ct * sa) + (ca * st);
  const R yy = sa * sb;
  const R dx = (cp * xx) - (sp * yy);
  const R dy = (cp * yy) + (sp * xx);
  const R dz = (ca * ct) - (cb * sa * st);
  theta = matan2(msqrt((dx * dx) + (dy * dy)), dz);
  phi = matan2(dy, dx);
}

// TabulatedInelasticSM.cu:153-207 with the constructor defaults (energy for
// ionisation = deltaE, default branching ratios)
template <typename R> CM_D R pick_be(const Mech& k, R deltaE) {
  if ((k.ncore > 0) && (deltaE <= (R)k.core[0])) return 0;
  int i = 0;
  while ((i < k.ncore) && ((R)k.core[i] <= deltaE)) ++i;
  if (i == 0) return 0;
  return (R)k.core[i - 1];
}

// TabulatedInelasticSM::scatter (TabulatedInelasticSM.cu:209-434).  d/E is
// the primary (updated in place); returns true with sd/sE set when a
// secondary is generated.  Deviates come in the reference's order.
template <typename R, typename G>
CM_D bool tabulated_scatter(const SceneView<R>& s, const Mech& k, R d[3], R& E, R sd[3], R& sE, G& g, R* theta_out = nullptr) {
  const R kE0 = E;
  const R kE = kE0 + (R)k.energyOffset;
  if (kE < (R)k.eiDomain0) return false;
  R theta = 0, phi = 0;
  R randoms[4];
  randoms[0] = g.next(); randoms[1] = g.next(); randoms[2] = g.next(); randoms[3] = g.next();
  R deltaE = kE * table_interp(s, k.tRed, kE, randoms[0], R(0), 3);
  const R gap = (R)k.energyGap, bandgap = (R)k.bandgap, oFE = (R)k.offsetFermiEnergy;
  if ((deltaE < gap) && (deltaE > (R(0.95) * gap))) deltaE = gap;
  const R d0[3] = {d[0], d[1], d[2]};
  if (deltaE >= bandgap) {
    R red = (deltaE - gap) / (kE - oFE - (R(2) * gap));
    if (red > R(1)) red = 1;
    else if (red < R(0)) red = 0;
    theta = table_interp(s, k.tTheta, kE, red, randoms[1], 3);
    if (theta_out) *theta_out = theta;
    phi = R(2) * R(kPi) * randoms[2];
    update_dir(d, theta, phi);
  }
  E = kE0 - deltaE;
  if (deltaE < bandgap) return false;
  R ct = mcos(theta);
  // momentum-transfer energy; in FP32 the reference's form loses everything to cancellation for small
  // losses and angles, so it is evaluated in double as (sqrt(E) - sqrt(E - dE))^2 + 4 sqrt(E (E - dE)) sin^2(theta/2)
  R Eq;
  if (sizeof(R) == 4) {
    const double a = sqrt((double)kE), b = sqrt((double)kE - (double)deltaE), sh = sin(0.5 * (double)theta);
    Eq = (R)(((a - b) * (a - b)) + (4.0 * a * b * sh * sh));
  } else {
    Eq = (R(2) * kE) - deltaE - (R(2) * msqrt(kE * (kE - deltaE)) * ct);
  }
  const R bEref = (R)k.bEref, ecb = (R)k.energyCBbottom, minGen = (R)k.minEgenSE, off = (R)k.energyOffset;
  R energySE;
  const R be = pick_be(k, deltaE);
  if (k.methodSE == 1 || k.methodSE == 2) {
    if (k.methodSE == 1 || be > 0) energySE = (deltaE + bEref) - be;
    else {
      R e0 = table_interp(s, k.tSEE0, deltaE, randoms[3], R(0), 3);
      if (e0 < (R)k.rangeSE0lo) e0 = (R)k.rangeSE0lo;
      else if (e0 > (R)k.rangeSE0hi) e0 = (R)k.rangeSE0hi;
      energySE = (deltaE + e0) - off;
    }
    if ((energySE + ecb) < minGen) return false;
    sd[0] = d0[0]; sd[1] = d0[1]; sd[2] = d0[2];
    update_dir(sd, R(kPi / 2) - theta, phi + R(kPi));
    sE = energySE;
    return true;
  }
  // methodSE 3
  if (be > 0) {  // core level: isotropic
    energySE = (deltaE + bEref) - be;
    if ((energySE + ecb) < minGen) return false;
    const R thetaSE = iso_angle(g.next());
    const R phiSE = R(2) * R(kPi) * g.next();
    dir_from_angles(sd, thetaSE, phiSE);
    sE = energySE;
    return true;
  }
  const R root = R(2) * msqrt(oFE * (oFE + deltaE));
  const R sum = (R(2) * oFE) + deltaE;
  const R Eqmin = sum - root, Eqmax = sum + root;
  if ((Eqmin <= Eq) && (Eq <= Eqmax)) {  // single electron: simESEf (TabulatedInelasticSM.cu:87-101)
    // in double in both precisions (a rare branch whose differences cancel in float)
    const double q = sqrt((double)Eq);
    const double kz = ((double)deltaE - (double)Eq) / 2. / q;
    const double kzf = kz + q;
    const double Ezq = kzf * kzf;
    double minE = ((double)oFE + (double)bandgap) - Ezq;
    if (minE < 0.) minE = 0;
    const double maxE = (double)oFE - (kz * kz);
    const double r = (double)randoms[3];
    const double Exy = (minE * (1. - r)) + (maxE * r);
    const double ESEf = Exy + Ezq;
    const R th1 = (R)acos(kzf / sqrt(ESEf));
    energySE = (R)(ESEf - (double)off);
    if ((energySE + ecb) < minGen) return false;
    R nth = R(kPi / 2) - theta, nph = phi + R(kPi);
    update_angles(nth, nph, th1, R(2) * R(kPi) * g.next());
    sd[0] = d0[0]; sd[1] = d0[1]; sd[2] = d0[2];
    update_dir(sd, nth, nph);
    sE = energySE;
    return true;
  }
  // plasmon: SE E0 table, isotropic
  R e0 = table_interp(s, k.tSEE0, deltaE, randoms[3], R(0), 3);
  if (e0 < (R)k.rangeSE0lo) e0 = (R)k.rangeSE0lo;
  else if (e0 > (R)k.rangeSE0hi) e0 = (R)k.rangeSE0hi;
  energySE = (deltaE + e0) - off;
  if ((energySE + ecb) < minGen) return false;
  const R thetaSE = iso_angle(g.next());
  const R phiSE = R(2) * R(kPi) * g.next();
  dir_from_angles(sd, thetaSE, phiSE);
  sE = energySE;
  return true;
}

// SelectableElasticSM::scatter (SelectableElasticSM.cu:49-67) at the step's
// starting energy Ep; returns the element picked.
template <typename R, typename G> CM_D int elastic_scatter(const SceneView<R>& s, const Mech& k, R d[3], R Ep, G& g) {
  const R u = g.next();
  int el = 0;
  if (k.nel > 1) {
    const R logE = mlog(Ep);
    R cum[kMaxElem];
    R tot = 0;
    for (int i = 0; i < k.nel; ++i) {
      tot += nistmott_rate(s, s.mott[k.mott[i]], k.mottMethod, (R)k.kel[i], (R)k.kbrown[i], Ep, logE);
      cum[i] = tot;
    }
    const R r = u * tot;
    while (el < k.nel - 1 && cum[el] < r) ++el;
  }
  const R alpha = nistmott_angle(s, s.mott[k.mott[el]], k.mottMethod, Ep, g);
  const R beta = R(2 * kPi) * g.next();
  update_dir(d, alpha, beta);
  return el;
}

// The deflection of GanachaudMokraniPhononInelasticSM::scatter (GanachaudMokraniPhononInelasticSM.cu:19-44)
// for x = hbar omega / E (with omx = 1 - x, both formed in double) and the deviate r0.  Double: the
// reference's cos(theta) as written.
template <typename R> CM_D R phonon_theta(double x, double omx, R r0);
template <> CM_D double phonon_theta(double x, double, double r0) {
  double costheta;
  if (x < 0.1) costheta = 1 + (((x * x) - (pow(16.0, r0) * pow(x, 2.0 - (2.0 * r0)))) / 8.0);
  else {
    const double root = sqrt(1.0 - x);
    const double temp = pow(((-2.0 * (1 + root)) + x) / ((-2.0 * (1 - root)) + x), r0);
    costheta = temp + (((x - 2.0) * (temp - 1)) / 2.0 / root);
  }
  return acos(costheta);
}
// Float: the angle in double as well.  Its exponent r0 ln(16/x^2) reaches ~20 for low-loss events, where
// the rounding of a float argument alone moves the angle by ~1e-6; phonon events are a small share of the
// steps, so the double evaluation costs little.
template <> CM_D float phonon_theta(double xd, double omxd, float r0) {
  return (float)phonon_theta<double>(xd, omxd, (double)r0);
}

// GanachaudMokraniPhononInelasticSM::scatter (GanachaudMokraniPhononInelasticSM.cu:19-44)
template <typename R, typename G> CM_D void phonon_scatter(const Mech& k, R d[3], R& E, R& Ep, G& g) {
  const R kE0 = E;
  // the threshold and the energy ratio in double, as in phonon_rate
  if ((double)kE0 < k.phononE) return;
  const double xd = k.phononE / (double)kE0;
  const R r0 = g.next(), r1 = g.next();
  const R phi = R(2) * R(kPi) * r1;
  update_dir(d, phonon_theta<R>(xd, ((double)kE0 - k.phononE) / (double)kE0, r0), phi);
  E = (R)((double)kE0 - k.phononE);
  Ep = kE0;
}

// ExpQMBarrierSM::barrierScatter (JMONSEL/ExpQMBarrierSM.cu:50-219).  The
// reference overwrites the struck surface normal with the direction of motion
// whenever the shape reports one (line 111-112); options bit 0 restores the
// normal (refraction).  hn is the struck boundary's outward normal from
// find_end_of_step.  Returns the region after the event.
template <typename R, typename G>
CM_D int barrier_scatter(const SceneView<R>& s, const Msm& m, double p[3], R d[3], R& E, int cur, int next, const double hn[3],
                         G& g) {
  if (cur == next) return cur;
  const Msm& curm = s.msms[s.regions[cur].msm];
  const Msm& nextm = s.msms[s.regions[next].msm];
  R deltaU = -(R)curm.ecb;
  if (!(deltaU == -(R)m.u0)) return cur;
  deltaU += (R)nextm.ecb;
  R nb[3];
  if (s.options & 1) {
    const R sign = is_containing_region(s, cur, next) ? R(-1) : R(1);
    nb[0] = sign * (R)hn[0]; nb[1] = sign * (R)hn[1]; nb[2] = sign * (R)hn[2];
  } else {
    nb[0] = d[0]; nb[1] = d[1]; nb[2] = d[2];
  }
  const R n0[3] = {d[0], d[1], d[2]};
  const R cosalpha = (n0[0] * nb[0]) + (n0[1] * nb[1]) + (n0[2] * nb[2]);
  if (cosalpha <= R(0)) {
    p[0] -= kSmallDispNm * (double)nb[0];
    p[1] -= kSmallDispNm * (double)nb[1];
    p[2] -= kSmallDispNm * (double)nb[2];
    return cur;
  }
  if (deltaU == R(0)) {
    p[0] += kSmallDispNm * (double)nb[0];
    p[1] += kSmallDispNm * (double)nb[1];
    p[2] += kSmallDispNm * (double)nb[2];
    return next;
  }
  const R kE0 = E;
  const R perpE = kE0 <= R(0) ? R(0) : cosalpha * cosalpha * kE0;
  R rootPerpE = 0, rootDiff = 0;
  bool transmits;
  if ((perpE == R(0)) || (perpE <= deltaU)) transmits = false;
  else {
    rootPerpE = msqrt(perpE);
    rootDiff = msqrt(perpE - deltaU);
    if (m.classical) transmits = true;
    else {
      R tp;
      if (m.lambda == 0.) {
        const R ksum = rootPerpE + rootDiff;
        tp = (R(4) * rootPerpE * rootDiff) / (ksum * ksum);
      } else {
        const R k1 = (R)m.lambdaFactor * rootPerpE;
        if (k1 > R(50)) tp = 1;
        else {
          const R k2 = (R)m.lambdaFactor * rootDiff;
          const R ratio = msinh(k1 - k2) / msinh(k1 + k2);
          tp = R(1) - (ratio * ratio);
        }
      }
      transmits = g.next() < tp;
    }
  }
  R nf[3];
  int out = cur;
  if (transmits) {
    const R factor = cosalpha * ((rootDiff / rootPerpE) - R(1));
    for (int i = 0; i < 3; i++) nf[i] = n0[i] + (factor * nb[i]);
    E = kE0 - deltaU;
    out = next;
    p[0] += kSmallDispNm * (double)nb[0];
    p[1] += kSmallDispNm * (double)nb[1];
    p[2] += kSmallDispNm * (double)nb[2];
  } else {
    const R two = R(2) * cosalpha;
    for (int i = 0; i < 3; i++) nf[i] = n0[i] - (nb[i] * two);
    p[0] -= kSmallDispNm * (double)nb[0];
    p[1] -= kSmallDispNm * (double)nb[1];
    p[2] -= kSmallDispNm * (double)nb[2];
  }
  // theta = acos(nf_z/|nf|), phi = atan2(nf_y, nf_x): the direction of nf
  const R inv = R(1) / msqrt(nf[0] * nf[0] + nf[1] * nf[1] + nf[2] * nf[2]);
  d[0] = nf[0] * inv; d[1] = nf[1] * inv; d[2] = nf[2] * inv;
  return out;
}

}  // namespace cm
