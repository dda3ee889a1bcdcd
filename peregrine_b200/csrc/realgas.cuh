// The cubic real gas and its double-flux tangent plane, device side.
//
// A generic two-parameter cubic, p = Ru T / (v - b) - a / (v^2 + u b v + w b^2),
// with the reference's mixing (kij = 0, sqrt(a) summed over mole fractions)
// and volume translation; the reference ships Soave-Redlich-Kwong, and
// Peng-Robinson is the same code on other constants
// (peregrine/simulator/mixture/eos/realgas/model.py:26-66).  Each function is
// the reference template's arithmetic, cited per function, on values in
// registers; the mixing sums take the reference's explicit fused
// multiply-adds.
#pragma once
#include "physics.cuh"

namespace pgb {

// the cubic at a point, passed between the steps (the reference's Cubic struct)
struct Cubic {
  double MWmix, bm, cm, S1, S2, am, dam, Astar, Bstar, Cstar, invRuT, Z, z1, z2, invslope, dZdT, v, I, logratio, q, qd;
};

// the real gas's mixture moments: the thermally perfect ones plus the
// cubic's covolume, translation and da sums per unit of Y_n / MW_n
// (peregrine/simulator/mixture/eos/realgas/model.py:13-14 through mixing.mako:3-30)
struct RGMom {
  double R, h298, b, c, da;
  double cc[MAXT];
};

template <int NS, class YF>
__device__ __forceinline__ RGMom mixmom_rg(YF Y) {
  RGMom m;
  m.R = m.h298 = m.b = m.c = m.da = 0.0;
#pragma unroll
  for (int t = 0; t < MAXT; t++) m.cc[t] = 0.0;
  double Ylast = 1.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double Yn = Y(n);
    Ylast -= Yn;
    m.R += Yn * kSp.Rsp[n];
    m.h298 += Yn * kSp.h298R[n];
    m.b += Yn * kSp.cbMW[n];
    m.c += Yn * kSp.vshiftMW[n];
    m.da += Yn * kSp.cdaMW[n];
#pragma unroll
    for (int t = 0; t < MAXT; t++)
      if (t < kSp.ncp) m.cc[t] += Yn * kSp.cppolyR[n * MAXT + t];
  }
  constexpr int L = NS - 1;
  m.R += Ylast * kSp.Rsp[L];
  m.h298 += Ylast * kSp.h298R[L];
  m.b += Ylast * kSp.cbMW[L];
  m.c += Ylast * kSp.vshiftMW[L];
  m.da += Ylast * kSp.cdaMW[L];
#pragma unroll
  for (int t = 0; t < MAXT; t++)
    if (t < kSp.ncp) m.cc[t] += Ylast * kSp.cppolyR[L * MAXT + t];
  return m;
}

// cubicmix (peregrine/simulator/mixture/eos/realgas/kernels/eos.mako:12-17)
__device__ __forceinline__ void cubicmix(Cubic &c, const RGMom &mom) {
  c.MWmix = kSp.Ru / mom.R;
  c.bm = mom.b * c.MWmix;
  c.cm = mom.c * c.MWmix;
  c.S2 = mom.da * c.MWmix;
}

// sqrt(a_n) per unit of Y_n / MW_n: Soave's modulus opened as
// |(1 + m) - sqrt(T) m / sqrt(Tc)| (eos.mako:5-8)
__device__ __forceinline__ double sqrtaMW(const int n, const double sqrtT) {
  return kSp.csqrtacMW[n] * fabs(fma(-sqrtT, kSp.cmTc[n], kSp.conepm[n]));
}
__device__ __forceinline__ double sqrta(const int n, const double sqrtT) {
  return kSp.csqrtac[n] * fabs(fma(-sqrtT, kSp.cmTc[n], kSp.conepm[n]));
}

// attraction: am = S1^2 and dam/dT = -S1 S2 / sqrt(T) (eos.mako:20-32)
template <int NS, class YF>
__device__ __forceinline__ void attraction(Cubic &c, YF Y, const double T) {
  const double sqrtT = sqrt(T);
  double s1 = 0.0, Ylast = 1.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double Yn = Y(n);
    Ylast -= Yn;
    s1 = fma(Yn, sqrtaMW(n, sqrtT), s1);
  }
  s1 = fma(Ylast, sqrtaMW(NS - 1, sqrtT), s1);
  c.S1 = s1 * c.MWmix;
  c.am = c.S1 * c.S1;
  c.dam = -c.S1 * c.S2 / sqrtT;
}

// dimless (eos.mako:34-43)
__device__ __forceinline__ void dimless(Cubic &c, const double p, const double T) {
  c.invRuT = 1.0 / (kSp.Ru * T);
  const double pRT = p * c.invRuT;
  c.Astar = c.am * pRT * c.invRuT;
  c.Bstar = c.bm * pRT;
  c.Cstar = c.cm * pRT;
  const double B = c.Bstar, B2 = B * B;
  c.z1 = c.Astar + kSp.cw * B2 - kSp.cu * B - kSp.cu * B2;
  c.z2 = -(1.0 + B - kSp.cu * B);
}

// rootslope (eos.mako:95-97)
__device__ __forceinline__ void rootslope(Cubic &c) { c.invslope = 1.0 / (3.0 * c.Z * c.Z + 2.0 * c.Z * c.z2 + c.z1); }

// zsolve: Cardano; of several roots above the covolume the least Gibbs
// energy departure's, the largest when none is (eos.mako:45-93)
__device__ __forceinline__ void zsolve(Cubic &c, const double p, const double T) {
  dimless(c, p, T);
  const double B = c.Bstar, B2 = B * B, z1 = c.z1, z2 = c.z2;
  const double z0 = -(c.Astar * B + kSp.cw * B2 * (1.0 + B));
  const double Q = (z2 * z2 - 3.0 * z1) * (1.0 / 9.0);
  const double R = (2.0 * z2 * z2 * z2 - 9.0 * z2 * z1 + 27.0 * z0) * (1.0 / 54.0);
  const double M = R * R - Q * Q * Q;
  const double z2o3 = z2 * (1.0 / 3.0);
  if (M > 0.0) {
    const double S = -copysign(cbrt(fabs(R) + sqrt(M)), R);
    c.Z = S + Q / S - z2o3;
  } else {
    const double sqQ = sqrt(Q), twopio3 = 2.0943951023931954923;
    const double theta3 = acos(R / (Q * sqQ)) * (1.0 / 3.0);
    const double roots[3] = {-2.0 * sqQ * cos(theta3) - z2o3, -2.0 * sqQ * cos(theta3 + twopio3) - z2o3,
                             -2.0 * sqQ * cos(theta3 - twopio3) - z2o3};
    double Z = fmax(roots[0], fmax(roots[1], roots[2]));
    int above = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) above += roots[k] > B;
    if (above > 1) {
      const double AoBse = c.Astar / (B * (kSp.csigma - kSp.ceps));
      double gmin = 0.0;
      bool found = false;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        const double z = roots[k];
        if (z <= B) continue;
        const double g = z - 1.0 - log(z - B) + AoBse * log((z + kSp.ceps * B) / (z + kSp.csigma * B));
        if (!found || g < gmin) {
          gmin = g;
          Z = z;
          found = true;
        }
      }
    }
    c.Z = Z;
  }
  rootslope(c);
}

// Z's derivative along (dA*, dB*) (eos.mako:99-105)
__device__ __forceinline__ double dZ(const Cubic &c, const double dAstar, const double dBstar) {
  const double B = c.Bstar, Z = c.Z, Z2 = Z * Z;
  const double dz0 = -(B * dAstar + (c.Astar + (2.0 * B + 3.0 * B * B) * kSp.cw) * dBstar);
  const double dz1 = dAstar + (2.0 * B * (kSp.cw - kSp.cu) - kSp.cu) * dBstar;
  const double dz2 = -(1.0 - kSp.cu) * dBstar;
  return -(dz2 * Z2 + dz1 * Z + dz0) * c.invslope;
}

// departures: h and cp residuals over R, the translation's -C* in h
// (eos.mako:108-122)
__device__ __forceinline__ void departures(double &hdep, double &cpdep, Cubic &c, const double T) {
  const double Tinv = kSp.Ru * c.invRuT;
  const double dlnamdT = c.dam / c.am;
  c.dZdT = dZ(c, -2.0 * c.Astar * Tinv * (1.0 - 0.5 * T * dlnamdT), -c.Bstar * Tinv);
  const double x = c.Z / c.Bstar, xm1 = x - 1.0;
  const double D = x * x + kSp.cu * x + kSp.cw;
  c.logratio = log((x + kSp.ceps) / (x + kSp.csigma));
  const double invBmRu = 1.0 / (c.bm * kSp.Ru);
  const double hres = invBmRu / (kSp.csigma - kSp.ceps) * (c.am * Tinv - c.dam) * c.logratio;
  c.qd = c.dam * invBmRu;
  c.q = c.am * invBmRu * Tinv;
  const double num = D - c.qd * xm1;
  cpdep = hres * 0.5 * T * dlnamdT + num * num / (D * D - c.q * (2.0 * x + kSp.cu) * xm1 * xm1) - 1.0;
  hdep = hres + (c.Z - 1.0) - c.Cstar;
}

// gamma and the speed of sound (eos.mako:124-137)
__device__ __forceinline__ void gamma_c(double &gamma, double &cs, const Cubic &c, const double p, const double T,
                                        const double rho, const double cp, const double invZt) {
  const double invp = 1.0 / p, Tinv = kSp.Ru * c.invRuT;
  const double dZtdT = c.dZdT + c.Cstar * Tinv;
  const double dZdp = dZ(c, c.Astar * invp, c.Bstar * invp);
  const double dZtdp = dZdp - c.Cstar * invp;
  const double drhodp = rho * invp * (1.0 - p * dZtdp * invZt);
  const double r = -Tinv * (1.0 + T * dZtdT * invZt);
  const double csq = 1.0 / (drhodp - (T / cp) * r * r);
  gamma = drhodp * csq;
  cs = sqrt(fabs(csq));
}

// the real gas's state with its root Z
struct RGState {
  State s;
  double Z;
};

// frompT (eos.mako:139-155)
template <int NS, class YF>
__device__ __forceinline__ RGState frompT_rg(const double p, const double T, YF Y) {
  const RGMom mom = mixmom_rg<NS>(Y);
  Cubic c;
  cubicmix(c, mom);
  attraction<NS>(c, Y, T);
  double cp_ideal, h_ideal;
  ideal_cph(mom.cc, mom.h298, T, cp_ideal, h_ideal);
  zsolve(c, p, T);
  double hdep, cpdep;
  departures(hdep, cpdep, c, T);
  RGState o;
  o.s.p = p;
  o.s.T = T;
  o.Z = c.Z;
  o.s.cp = cp_ideal + mom.R * cpdep;
  const double Zt = c.Z - c.Cstar, invZt = 1.0 / Zt, porho = Zt * mom.R * T;
  o.s.rho = p * c.invRuT * c.MWmix * invZt;
  o.s.rhoinv = 1.0 / o.s.rho;
  o.s.e = h_ideal + mom.R * T * hdep - porho;
  gamma_c(o.s.gamma, o.s.c, c, p, T, o.s.rho, o.s.cp, invZt);
  return o;
}

// atvolume (eos.mako:157-160)
__device__ __forceinline__ void atvolume(Cubic &c, const double rho) {
  c.v = c.MWmix / rho + c.cm;
  c.I = log((c.v + kSp.csigma * c.bm) / (c.v + kSp.ceps * c.bm)) / ((kSp.csigma - kSp.ceps) * c.bm);
}

// fromrhoE: Newton in T at the cell's volume from its last T, then the state
// there, Z the volume's (eos.mako:162-190, realgas/kernels/newton.mako:3-14)
template <int NS, class YF>
__device__ __forceinline__ RGState fromrhoE_rg(const RGMom &mom, YF Y, const double rho, const double e,
                                               const double Tguess) {
  Cubic c;
  cubicmix(c, mom);
  atvolume(c, rho);
  const double invMWmix = 1.0 / c.MWmix;
  double T = (Tguess < 1.0) ? 300.0 : Tguess;
  double cp_ideal, h_ideal;
  const double tol = 1e5 * 2.220446049250313e-16;
  for (int k = 0; k < 12; k++) {
    attraction<NS>(c, Y, T);
    ideal_cph(mom.cc, mom.h298, T, cp_ideal, h_ideal);
    const double app = 0.5 * (c.S2 * c.S2 - c.dam) / T;
    const double f = h_ideal - mom.R * T - (c.am - T * c.dam) * c.I * invMWmix - e;
    const double cv = cp_ideal - mom.R + T * app * c.I * invMWmix;
    const double dT = f / cv;
    T -= dT;
    if (k >= 2 && fabs(dT) <= tol * T) break;
  }
  attraction<NS>(c, Y, T);
  ideal_cph(mom.cc, mom.h298, T, cp_ideal, h_ideal);
  const double vs = c.v + kSp.csigma * c.bm, ve = c.v + kSp.ceps * c.bm;
  const double p = kSp.Ru * T / (c.v - c.bm) - c.am / (vs * ve);
  dimless(c, p, T);
  c.Z = p * c.invRuT * c.v;
  rootslope(c);
  double hdep, cpdep;
  departures(hdep, cpdep, c, T);
  RGState o;
  o.s.rho = rho;
  o.s.rhoinv = 1.0 / rho;
  o.s.e = e;
  o.s.p = p;
  o.s.T = T;
  o.Z = c.Z;
  o.s.cp = cp_ideal + mom.R * cpdep;
  const double invZt = 1.0 / (c.Z - c.Cstar);
  gamma_c(o.s.gamma, o.s.c, c, p, T, rho, o.s.cp, invZt);
  return o;
}

// fromrhop: the double flux's state at the plane's pressure, Newton in T at
// the cell's volume (realgasdf/kernels/eos.mako:6-30, realgasdf/kernels/newton.mako:3-13)
template <int NS, class YF>
__device__ __forceinline__ RGState fromrhop_rg(const RGMom &mom, YF Y, const double rho, const double p,
                                               const double Tguess) {
  Cubic c;
  cubicmix(c, mom);
  atvolume(c, rho);
  const double vs = c.v + kSp.csigma * c.bm, ve = c.v + kSp.ceps * c.bm;
  const double invvmb = 1.0 / (c.v - c.bm), invD = 1.0 / (vs * ve);
  double T = (Tguess < 1.0) ? 300.0 : Tguess;
  const double tol = 1e5 * 2.220446049250313e-16;
  for (int k = 0; k < 12; k++) {
    attraction<NS>(c, Y, T);
    const double f = kSp.Ru * T * invvmb - c.am * invD - p;
    const double dpdT = kSp.Ru * invvmb - c.dam * invD;
    const double dT = f / dpdT;
    T -= dT;
    if (k >= 2 && fabs(dT) <= tol * T) break;
  }
  attraction<NS>(c, Y, T);
  double cp_ideal, h_ideal;
  ideal_cph(mom.cc, mom.h298, T, cp_ideal, h_ideal);
  dimless(c, p, T);
  c.Z = p * c.invRuT * c.v;
  rootslope(c);
  double hdep, cpdep;
  departures(hdep, cpdep, c, T);
  RGState o;
  o.s.rho = rho;
  o.s.rhoinv = 1.0 / rho;
  o.s.p = p;
  o.s.T = T;
  o.Z = c.Z;
  o.s.cp = cp_ideal + mom.R * cpdep;
  o.s.e = h_ideal + mom.R * T * hdep - p / rho;
  const double invZt = 1.0 / (c.Z - c.Cstar);
  gamma_c(o.s.gamma, o.s.c, c, p, T, rho, o.s.cp, invZt);
  return o;
}

// the species' partial enthalpies at a stored state (p, T, Z): hspecies with
// hpartialpoint and hpartial (eos.mako:192-224, 257-273)
template <int NS, class YF>
__device__ __forceinline__ void hspecies_rg(double *h, const RGMom &mom, YF Y, const double p, const double T,
                                            const double Z) {
  Cubic c;
  cubicmix(c, mom);
  attraction<NS>(c, Y, T);
  dimless(c, p, T);
  c.Z = Z;
  rootslope(c);
  double hdep, cpdep;
  departures(hdep, cpdep, c, T);
  // hpartialpoint
  const double lnT = log(T), Tinv = kSp.Ru * c.invRuT, sqrtT = sqrt(T);
  const double B = c.Bstar, ZT = c.dZdT, BT = -B * Tinv;
  const double invZsB = 1.0 / (Z + kSp.csigma * B), invZeB = 1.0 / (Z + kSp.ceps * B);
  const double Iz = -c.logratio / (kSp.csigma - kSp.ceps);
  const double IzT = ((ZT + kSp.csigma * BT) * invZsB - (ZT + kSp.ceps * BT) * invZeB) / (kSp.csigma - kSp.ceps);
  const double dlnZmB = (ZT - BT) / (Z - B);
  const double invS1 = 1.0 / c.S1, invBm = 1.0 / c.bm;
  const double invamsqrtT = invS1 * invS1 / sqrtT;
  const double qT = (c.qd - c.q) * Tinv;
#pragma unroll
  for (int n = 0; n < NS; n++) {
    double hRT = 0.0;
#pragma unroll
    for (int m = MAXT - 1; m >= 0; m--)
      if (m < kSp.nh) hRT = hRT * lnT + kSp.hpoly[n * MAXT + m];
    hRT += kSp.h298[n] * Tinv;
    const double sqrtan = sqrta(n, sqrtT);
    const double r = 2.0 * sqrtan * invS1;
    const double rT = (sqrtan * c.S2 - kSp.cda[n] * c.S1) * invamsqrtT;
    const double bb = kSp.cb[n] * invBm;
    const double qbar = c.q * (r - bb), qbarT = qT * (r - bb) + c.q * rT;
    const double dlnphidT = bb * c.dZdT - dlnZmB - qbarT * Iz - qbar * IzT;
    h[n] = (hRT * T * kSp.Ru - kSp.Ru * T * T * dlnphidT - kSp.vshift[n] * p) * kSp.MWinv[n];
  }
}

// drho: the density's derivatives in p, T and the carried Y at fixed others
// (eos.mako:226-255)
template <int NS, class YF>
__device__ __forceinline__ void drho_rg(double &rho_p, double &rho_T, double *rho_Y, const RGMom &mom, YF Y,
                                        const double p, const double T, const double rho) {
  Cubic c;
  cubicmix(c, mom);
  attraction<NS>(c, Y, T);
  zsolve(c, p, T);
  double hdep, cpdep;
  departures(hdep, cpdep, c, T);
  const double invp = 1.0 / p, Tinv = kSp.Ru * c.invRuT, sqrtT = sqrt(T);
  const double Zt = c.Z - c.Cstar, dZtdT = c.dZdT + c.Cstar * Tinv, invZt = 1.0 / Zt;
  const double dZdp = dZ(c, c.Astar * invp, c.Bstar * invp);
  rho_p = rho * invp * (1.0 - (p * dZdp - c.Cstar) * invZt);
  rho_T = -rho * Tinv * (1.0 + T * dZtdT * invZt);
  const double twoS1 = 2.0 * c.S1;
  const double invRuT = Tinv / kSp.Ru, pRT = p * invRuT;
  const double MWinv_last = kSp.MWinv[NS - 1];
  const double sqrta_last = sqrtaMW(NS - 1, sqrtT);
  const double b_last = kSp.cbMW[NS - 1], c_last = kSp.vshiftMW[NS - 1];
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double dlnMWmix = -c.MWmix * (kSp.MWinv[n] - MWinv_last);
    const double dam = twoS1 * (c.S1 * dlnMWmix + c.MWmix * (sqrtaMW(n, sqrtT) - sqrta_last));
    const double dbm = c.bm * dlnMWmix + c.MWmix * (kSp.cbMW[n] - b_last);
    const double dcm = c.cm * dlnMWmix + c.MWmix * (kSp.vshiftMW[n] - c_last);
    const double dZdY = dZ(c, dam * pRT * invRuT, dbm * pRT);
    rho_Y[n] = rho * (dlnMWmix - (dZdY - dcm * pRT) * invZt);
  }
}

// planeslopes: theta and eps + sum zeta Y of the tangent plane of rho e
// (realgasdf/kernels/eos.mako:32-48)
template <int NS, class YF>
__device__ __forceinline__ void planeslopes(double &theta, double &epsY, const RGMom &mom, YF Y, const double rho,
                                            const double rhoinv, const double T, const double e) {
  Cubic c;
  cubicmix(c, mom);
  atvolume(c, rho);
  attraction<NS>(c, Y, T);
  const double vs = c.v + kSp.csigma * c.bm, ve = c.v + kSp.ceps * c.bm;
  const double invvmb = 1.0 / (c.v - c.bm), invD = 1.0 / (vs * ve), invMWmix = 1.0 / c.MWmix;
  double cp_ideal, h_ideal;
  ideal_cph(mom.cc, mom.h298, T, cp_ideal, h_ideal);
  const double app = 0.5 * (c.S2 * c.S2 - c.dam) / T;
  const double cv = cp_ideal - mom.R + T * app * c.I * invMWmix;
  const double p = kSp.Ru * T * invvmb - c.am * invD;
  const double dpdT = kSp.Ru * invvmb - c.dam * invD;
  const double dpdrho = c.MWmix * rhoinv * rhoinv * (kSp.Ru * T * invvmb * invvmb - c.am * (vs + ve) * invD * invD);
  theta = rho * cv / dpdT;
  epsY = e - (T * dpdT - p) * rhoinv - theta * dpdrho;
}

template <int NS, class YF>
__device__ __forceinline__ State frompT_rg_state(const double p, const double T, YF Y) {
  return frompT_rg<NS>(p, T, Y).s;
}

template <int NS, class YF>
__device__ __forceinline__ void hspecies_rg_of(double *h, YF Y, const double p, const double T, const double Z) {
  const RGMom mom = mixmom_rg<NS>(Y);
  hspecies_rg<NS>(h, mom, Y, p, T, Z);
}

}  // namespace pgb
