// Cell and face physics of the calorically perfect gas, device side.
//
// Each function is the reference template's arithmetic (cited per function),
// on values in registers; the callers decide where the values come from
// (global arrays on the per-block path, shared-memory planes on the fused
// path).  nvcc contracts multiply-adds as the reference's NVRTC build does
// (peregrine/backend/cuda/compiler.py:17).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace pgb {

constexpr int MAXNS = 12;
constexpr int MAXT = 8;  // terms of a fit in ln T

// the case's species tables, in constant memory; filled per case before its
// launches (a case's tables are copied in when the case is made current).
// Static: each translation unit of the library has its own copy and fills it.
struct Species {
  int ns;
  double Ru;
  double Rsp[MAXNS], cp0[MAXNS], h298R[MAXNS], MWinv[MAXNS], hpoly0[MAXNS], h298[MAXNS];
  double mu0[MAXNS], kappa0[MAXNS], MWqinv[MAXNS], lewis[MAXNS];
  double wilkepair[MAXNS * MAXNS];
  double alpha;
  // single-species shortcuts, exact copies of what the per-cell formulas give
  // for Y = 1 (set by the host from the same operations)
  double R1, cp1, h2981, cv1, cvinv1, gamma1, th1;  // th1 = cp / gamma
  double mu1, kappa1;
  // the thermally perfect gas and kinetic-theory transport: 0 / 1 selectors,
  // and fits in ln T, [species][term]: cp (times R_sp), h over R T, sqrt(mu)
  // over T^(1/4), kappa over sqrt(T) (peregrine/simulator/mixture/eos/tpg/model.py:7-9,
  // peregrine/simulator/mixture/transport/kinetic.py)
  int tpg, kinetic;
  int ncp, nh, nmu, nkappa;
  double cppolyR[MAXNS * MAXT], hpoly[MAXNS * MAXT], mupoly[MAXNS * MAXT], kappapoly[MAXNS * MAXT];
  // the sub-stepped chemistry's species heat capacities, cp / R_sp in ln T
  // (peregrine/simulator/mixture/eos/base.py:33-47), and molar masses
  int ncppoly;
  double cppoly[MAXNS * MAXT], MW[MAXNS];
  // binary diffusion (peregrine/simulator/mixture/diffusion/binary.py): the
  // pair fits of T^(3/2) / D at unit pressure, a row per species of its
  // partners' in walk order ([species][partner][term]), each species' own
  // pair, and the bath (a partial bath lists its species; width partners)
  int binary, bpartial, bwidth, npair, nself;
  int bath[MAXNS];
  // Herning's viscosity mixing rule in place of Wilke's
  // (peregrine/simulator/mixture/mixrule/herning.py): sqrt(MW) per species
  int herning;
  double sqrtMW[MAXNS];
  double pairfit[MAXNS * MAXNS * MAXT], selffit[MAXNS * MAXT];
  // the cubic real gas (a thermally perfect gas underneath, tpg set too) and
  // its double flux: the form's u, w and roots sigma, eps; per species
  // sqrt(a_c), b, -(da/dT) sqrt(T / a), m / sqrt(Tc), 1 + m, each of the first
  // three and the translation also per unit of 1 / MW
  // (peregrine/simulator/mixture/eos/realgas/model.py:43-98)
  int realgas, df;
  double cu, cw, csigma, ceps;
  double csqrtac[MAXNS], cb[MAXNS], cda[MAXNS], cmTc[MAXNS], conepm[MAXNS], vshift[MAXNS];
  double csqrtacMW[MAXNS], cbMW[MAXNS], cdaMW[MAXNS], vshiftMW[MAXNS];
};

static __constant__ Species kSp;

// The species tables, in the order the C ABI passes them packed, into the
// constant struct; and the single-species shortcuts by the same operations
// the per-cell formulas take for Y = 1 (mixmom gives R = 0 + 1 Rsp exactly,
// likewise cp and h298; transport.mako with X = MWinv / MWinv).
enum { T_RSP = 0, T_CP0, T_H298R, T_MWINV, T_HPOLY0, T_H298, T_MU0, T_KAPPA0, T_MWQINV, T_LEWIS, T_NTAB };
inline void species_fill(Species &s, int ns, double alpha, bool constant_transport, const double *const tab[T_NTAB],
                         const double *wilkepair) {
  s.ns = ns;
  s.alpha = alpha;
  s.Ru = 8314.46261815324;
  double *dst[T_NTAB] = {s.Rsp, s.cp0, s.h298R, s.MWinv, s.hpoly0, s.h298, s.mu0, s.kappa0, s.MWqinv, s.lewis};
  for (int q = 0; q < T_NTAB; q++)
    for (int n = 0; n < ns; n++) dst[q][n] = tab[q] ? tab[q][n] : 1.0;
  for (int n = 0; n < ns; n++)
    for (int m = 0; m < ns; m++) s.wilkepair[n * MAXNS + m] = wilkepair ? wilkepair[n * ns + m] : 0.25;
  s.R1 = 0.0 + 1.0 * s.Rsp[0];
  s.cp1 = 0.0 + 1.0 * s.cp0[0];
  s.h2981 = 0.0 + 1.0 * s.h298R[0];
  s.cv1 = s.cp1 - s.R1;
  s.cvinv1 = 1.0 / s.cv1;
  s.gamma1 = s.cp1 / s.cv1;
  s.th1 = s.cp1 / s.gamma1;
  s.mu1 = s.kappa1 = 0.0;
  s.tpg = s.kinetic = 0;
  s.ncp = s.nh = s.nmu = s.nkappa = 0;
  s.realgas = s.df = 0;
  if (ns == 1 && constant_transport) {
    volatile double Y = 1.0;
    const double denom = 0.0 + Y * s.MWinv[0];
    const double MWmix = 1.0 / denom;
    const double X = Y * s.MWinv[0] * MWmix;
    const double sqrtmu = std::sqrt(s.mu0[0]);
    const double sinv = 1.0 / (sqrtmu * s.MWqinv[0]);
    const double sn = sqrtmu * s.MWqinv[0];
    const double r = 1.0 + sn * sinv;
    const double phi = 0.0 + r * r * s.wilkepair[0] * X;
    s.mu1 = 0.0 + sqrtmu * sqrtmu * X / phi;
    const double series = 0.0 + X * s.kappa0[0];
    const double parallel = 0.0 + X / s.kappa0[0];
    s.kappa1 = 0.5 * (series + 1.0 / parallel);
  }
}

// a fit table [ns][terms] into the constant struct's [species][MAXT]
inline void fit_fill(double *dst, int &nterms, const double *src, int ns, int terms) {
  nterms = terms;
  for (int n = 0; n < ns; n++)
    for (int t = 0; t < MAXT; t++) dst[n * MAXT + t] = t < terms ? src[n * terms + t] : 0.0;
}

// EosState (peregrine/simulator/mixture/eos/base.py:85-86)
struct State {
  double p, T, rhoinv, rho, e, cp, gamma, c;
};

// mixmom for the cpg moments (peregrine/simulator/mixture/eos/kernels/mixing.mako:3-30)
template <int NS, class YF>
__device__ __forceinline__ void mixmom(YF Y, double &R, double &cp, double &h298) {
  R = 0.0, cp = 0.0, h298 = 0.0;
  double Ylast = 1.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double Yn = Y(n);
    Ylast -= Yn;
    R += Yn * kSp.Rsp[n];
    cp += Yn * kSp.cp0[n];
    h298 += Yn * kSp.h298R[n];
  }
  R += Ylast * kSp.Rsp[NS - 1];
  cp += Ylast * kSp.cp0[NS - 1];
  h298 += Ylast * kSp.h298R[NS - 1];
}

// the thermally perfect moments: R, h298 and cp's coefficients in ln T, each
// Y-weighted (peregrine/simulator/mixture/eos/kernels/mixing.mako:3-30 with
// the moments of peregrine/simulator/mixture/eos/tpg/model.py:7-9)
template <int NS, class YF>
__device__ __forceinline__ void mixmom_tpg(YF Y, double &R, double &h298, double *cc) {
  R = 0.0, h298 = 0.0;
#pragma unroll
  for (int t = 0; t < MAXT; t++) cc[t] = 0.0;
  double Ylast = 1.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double Yn = Y(n);
    Ylast -= Yn;
    R += Yn * kSp.Rsp[n];
    h298 += Yn * kSp.h298R[n];
#pragma unroll
    for (int t = 0; t < MAXT; t++)
      if (t < kSp.ncp) cc[t] += Yn * kSp.cppolyR[n * MAXT + t];
  }
  R += Ylast * kSp.Rsp[NS - 1];
  h298 += Ylast * kSp.h298R[NS - 1];
#pragma unroll
  for (int t = 0; t < MAXT; t++)
    if (t < kSp.ncp) cc[t] += Ylast * kSp.cppolyR[(NS - 1) * MAXT + t];
}

// ideal_cph: cp and h per mass at T from the moments, h's coefficients built
// from cp's in the same descent
// (peregrine/simulator/mixture/caloric/tdepcp/kernels/caloric.mako:4-15)
__device__ __forceinline__ void ideal_cph(const double *cc, const double h298, const double T, double &cp, double &h) {
  const double u = log(T);
  cp = 0.0;
  h = 0.0;
  double hcoeff = 0.0;
#pragma unroll
  for (int m = MAXT - 1; m >= 0; m--) {
    if (m < kSp.ncp) {
      cp = cp * u + cc[m];
      hcoeff = cc[m] - (m + 1) * hcoeff;
      h = h * u + hcoeff;
    }
  }
  h = h * T + h298;
}

// fromQ (peregrine/simulator/euler/kernels/state/fromQ.mako:5-19) with the
// calorically perfect fromrhoE (peregrine/simulator/mixture/eos/cpg/kernels/eos.mako:5-15)
// or the thermally perfect one: Newton from the cell's last T (300 K below
// 1 K), at least three steps and at most twelve, done once a step is within
// 1e5 eps of T; cp is left at the T before the last step
// (peregrine/simulator/mixture/eos/tpg/kernels/eos.mako:8-20,
//  peregrine/simulator/mixture/eos/tpg/kernels/newton.mako:3-10)
template <int NS, class QF>
__device__ __forceinline__ State fromQ(QF Q, const double Tguess = 0.0) {
  const double rho = Q(0), rhoinv = 1.0 / rho;
  const double q1 = Q(1), q2 = Q(2), q3 = Q(3);
  const double e = (Q(4) - 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) * rhoinv) * rhoinv;
  State s;
  if (kSp.tpg) {
    double R, h298, cc[MAXT];
    mixmom_tpg<NS>([&](int n) { return Q(5 + n) * rhoinv; }, R, h298, cc);
    double T = (Tguess < 1.0) ? 300.0 : Tguess;
    double cp = 0.0, h = 0.0;
    const double tol = 1e5 * 2.220446049250313e-16;
    for (int k = 0; k < 12; k++) {
      ideal_cph(cc, h298, T, cp, h);
      const double dT = (e - (h - R * T)) / (cp - R);
      T += dT;
      if (k >= 2 && fabs(dT) <= tol * T) break;
    }
    s.rho = rho;
    s.rhoinv = 1.0 / rho;
    s.e = e;
    s.T = T;
    s.p = rho * R * T;
    s.cp = cp;
    s.gamma = cp / (cp - R);
    s.c = sqrt(s.gamma * R * T);
    return s;
  }
  double R, cp, h298;
  mixmom<NS>([&](int n) { return Q(5 + n) * rhoinv; }, R, cp, h298);
  const double cv = cp - R;
  s.rho = rho;
  s.rhoinv = 1.0 / rho;
  s.e = e;
  s.T = (e - h298) / cv;
  s.p = rho * R * s.T;
  s.cp = cp;
  s.gamma = cp / cv;
  s.c = sqrt(s.gamma * R * s.T);
  return s;
}

// the real gas's frompT, in realgas.cuh
template <int NS, class YF>
__device__ __forceinline__ State frompT_rg_state(const double p, const double T, YF Y);

// RG: the case's gas is the cubic real gas.  A compile-time switch, so the
// ideal gases' kernels carry none of its registers.

// frompT: the calorically perfect (peregrine/simulator/mixture/eos/cpg/kernels/eos.mako:17-27),
// the thermally perfect (peregrine/simulator/mixture/eos/tpg/kernels/eos.mako:22-32)
// or the real gas (realgas.cuh)
template <int NS, class YF, bool RG = false>
__device__ __forceinline__ State frompT(const double p, const double T, YF Y) {
  if (RG) return frompT_rg_state<NS>(p, T, Y);
  State s;
  s.p = p;
  s.T = T;
  if (kSp.tpg) {
    double R, h298, cc[MAXT], cp, h;
    mixmom_tpg<NS>(Y, R, h298, cc);
    ideal_cph(cc, h298, T, cp, h);
    s.rho = p / (R * T);
    s.rhoinv = 1.0 / s.rho;
    s.e = h - R * T;
    s.cp = cp;
    s.gamma = cp / (cp - R);
    s.c = sqrt(s.gamma * R * T);
    return s;
  }
  double R, cp, h298;
  mixmom<NS>(Y, R, cp, h298);
  const double cv = cp - R;
  s.rho = p / (R * T);
  s.rhoinv = 1.0 / s.rho;
  s.e = cv * T + h298;
  s.cp = cp;
  s.gamma = cp / cv;
  s.c = sqrt(s.gamma * R * T);
  return s;
}

// fromprims (peregrine/simulator/euler/kernels/state/fromprims.mako:4-12,
// peregrine/simulator/euler/kernels/solution.mako:2-23 through the eos's
// frompT); the state it stores is returned
template <int NS>
__device__ __forceinline__ State fromprims(const double *q, double *Q) {
  const State th = frompT<NS>(q[0], q[4], [&](int n) { return q[5 + n]; });
  const double rho = th.rho;
  Q[0] = rho;
  Q[1] = rho * q[1];
  Q[2] = rho * q[2];
  Q[3] = rho * q[3];
  Q[4] = rho * (th.e + 0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
#pragma unroll
  for (int n = 0; n < NS - 1; n++) Q[5 + n] = rho * q[5 + n];
  return th;
}

// transport with constant species properties, Wilke, series/parallel
// conductivity, Lewis diffusivities and species enthalpies
// (peregrine/simulator/navstokes/kernels/transport.mako:5-35,
//  peregrine/simulator/mixture/transport/kernels/constant.mako:5-16,
//  peregrine/simulator/mixture/mixrule/kernels/wilke.mako:3-17,
//  peregrine/simulator/mixture/transport/kernels/mixing.mako:3-10,
//  peregrine/simulator/mixture/diffusion/kernels/lewis.mako:3-8,
//  peregrine/simulator/mixture/eos/kernels/species.mako:9-36)
template <int NS, class YF>
__device__ __forceinline__ void hspecies_rg_of(double *h, YF Y, const double p, const double T, const double Z);

// the mixture-averaged diffusion coefficients from the pair fits
// (peregrine/simulator/mixture/diffusion/kernels/binary.mako:13-62): per
// species the sums over its partners of X_m / D_nm and X_m MW_m / D_nm, one
// quotient; a species alone (X_n within 64 eps of one) takes its
// self-diffusion coefficient, a composition of nothing D = 0
template <int NS>
__device__ __forceinline__ void binary_diffusion(double *D, const double p, const double T, const double lnT,
                                                 const double *X) {
  const double invT32 = 1.0 / (T * sqrt(T));
  const double tiny = 64 * 2.220446049250313e-16;
  const int width = kSp.bwidth;
#pragma unroll
  for (int n = 0; n < NS; n++) {
    double sum1 = 0.0, sum2 = 0.0, rest = 0.0, bathx = 0.0;
    auto partner = [&](const int k, const int m, const double Xm) {
      double Dinv = 0.0;
#pragma unroll
      for (int t = MAXT - 1; t >= 0; t--)
        if (t < kSp.npair) Dinv = Dinv * lnT + kSp.pairfit[(n * MAXNS + k) * MAXT + t];
      Dinv *= invT32 * 1.0;
      sum1 += Xm * Dinv;
      sum2 += Xm * kSp.MW[m] * Dinv;
      rest += Xm * kSp.MW[m];
      bathx += Xm;
    };
    if (kSp.bpartial) {
      for (int k = 0; k < width; k++) {
        const int m = kSp.bath[k];
        double Xm = 0.0;
#pragma unroll
        for (int q = 0; q < NS; q++)
          if (q == m && m != n) Xm = fmax(X[q], 0.0);
        partner(k, m, Xm);
      }
    } else {
#pragma unroll
      for (int k = 0; k < NS - 1; k++) {
        const int m = k + (k >= n);
        partner(k, m, fmax(X[m], 0.0));
      }
    }
    double Dinvself = 0.0;
#pragma unroll
    for (int t = MAXT - 1; t >= 0; t--)
      if (t < kSp.nself) Dinvself = Dinvself * lnT + kSp.selffit[n * MAXT + t];
    Dinvself *= invT32 * 1.0;
    const double Xn = fmax(X[n], 0.0);
    bool alone;
    double num, den;
    if (kSp.bpartial) {
      alone = 1.0 - Xn <= tiny || bathx <= tiny;
      num = alone ? 1.0 : rest * bathx;
      den = alone ? p * Dinvself : p * ((1.0 - Xn) * rest * sum1 + Xn * bathx * sum2);
    } else {
      alone = 1.0 - Xn <= tiny;
      num = alone ? 1.0 : rest;
      den = alone ? p * Dinvself : p * (rest * sum1 + Xn * sum2);
    }
    D[n] = (alone || (rest > 0.0 && den > 0.0)) ? num / den : 0.0;
  }
}

template <int NS, class QF, bool RG = false>
__device__ __forceinline__ void transport(QF Q, const State &st, double *tr, double *hsp, const double Z = 0.0) {
  const double rho = Q(0), rhoinv = 1.0 / rho;
  double Ylast = 1.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) Ylast -= Q(5 + n) * rhoinv;
  Ylast = fmax(Ylast, 0.0);
  auto Y = [&](int n) { return n < NS - 1 ? Q(5 + n) * rhoinv : Ylast; };
  double denom = 0.0;
#pragma unroll
  for (int n = 0; n < NS; n++) denom += Y(n) * kSp.MWinv[n];
  const double MWmix = 1.0 / denom;
  double X[NS];
#pragma unroll
  for (int n = 0; n < NS; n++) X[n] = Y(n) * kSp.MWinv[n] * MWmix;
  double sqrtmu[NS], sinv[NS], kappasp[NS];
  const double T = st.T, lnT = log(T);
  if (kSp.kinetic) {
    // dilute kinetic theory (peregrine/simulator/mixture/transport/kernels/dilute.mako:5-26)
    const double sqrtT = sqrt(T), sqrtsqrtT = sqrt(sqrtT);
#pragma unroll
    for (int n = 0; n < NS; n++) {
      double fit = 0.0, fk = 0.0;
#pragma unroll
      for (int m = MAXT - 1; m >= 0; m--) {
        if (m < kSp.nmu) fit = fit * lnT + kSp.mupoly[n * MAXT + m];
        if (m < kSp.nkappa) fk = fk * lnT + kSp.kappapoly[n * MAXT + m];
      }
      sqrtmu[n] = fit * sqrtsqrtT;
      kappasp[n] = fk * sqrtT;
    }
  } else {
#pragma unroll
    for (int n = 0; n < NS; n++) sqrtmu[n] = sqrt(kSp.mu0[n]), kappasp[n] = kSp.kappa0[n];
  }
#pragma unroll
  for (int n = 0; n < NS; n++) sinv[n] = 1.0 / (sqrtmu[n] * kSp.MWqinv[n]);
  double mu = 0.0;
  if (kSp.herning) {
    // peregrine/simulator/mixture/mixrule/kernels/herning.mako:3-12
    double num = 0.0, den = 0.0;
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const double w = X[n] * kSp.sqrtMW[n];
      num += w * sqrtmu[n] * sqrtmu[n];
      den += w;
    }
    mu = num / den;
  } else {
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const double sn = sqrtmu[n] * kSp.MWqinv[n];
      double phi = 0.0;
#pragma unroll
      for (int m = 0; m < NS; m++) {
        const double r = 1.0 + sn * sinv[m];
        phi += r * r * kSp.wilkepair[n * MAXNS + m] * X[m];
      }
      mu += sqrtmu[n] * sqrtmu[n] * X[n] / phi;
    }
  }
  double series = 0.0, parallel = 0.0;
#pragma unroll
  for (int n = 0; n < NS; n++) {
    series += X[n] * kappasp[n];
    parallel += X[n] / kappasp[n];
  }
  const double kappa = 0.5 * (series + 1.0 / parallel);
  tr[0] = mu;
  tr[1] = kappa;
  if (kSp.binary) {
    binary_diffusion<NS>(tr + 2, st.p, T, lnT, X);
  } else {
    const double kor = kappa * rhoinv / st.cp;
#pragma unroll
    for (int n = 0; n < NS; n++) tr[2 + n] = kor / kSp.lewis[n];
  }
  // hspecies: the real gas's partial enthalpies at the stored state, or the
  // ideal ones (peregrine/simulator/mixture/eos/kernels/species.mako:9-15, 31-36)
  if (RG) {
    hspecies_rg_of<NS>(hsp, [&](int n) { return Q(5 + n) * rhoinv; }, st.p, T, Z);
    return;
  }
  const double u = lnT, Tinv = 1.0 / T;
#pragma unroll
  for (int n = 0; n < NS; n++) {
    double hRT = 0.0;
    if (kSp.nh > 0) {
#pragma unroll
      for (int m = MAXT - 1; m >= 0; m--)
        if (m < kSp.nh) hRT = hRT * u + kSp.hpoly[n * MAXT + m];
    } else {
      hRT = kSp.hpoly0[n];
    }
    hRT += kSp.h298[n] * Tinv;
    hsp[n] = hRT * T * kSp.Ru * kSp.MWinv[n];
  }
}

// A face side for kepaec: what the two-point flux reads of a cell
// (peregrine/simulator/euler/kernels/flux/recon/constant.mako:3-18)
struct KSide {
  double u, v, w, p, rho, e, th;  // th = cp / gamma * T
};

// kepaec (peregrine/simulator/euler/kernels/flux/function/kepaec.mako:2-20);
// the species rows are added by the caller
__device__ __forceinline__ void kepaec(const KSide &L, const KSide &R, const double S0, const double S1,
                                       const double S2, double *F, double &C) {
  const double uf = 0.5 * (R.u + L.u), vf = 0.5 * (R.v + L.v), wf = 0.5 * (R.w + L.w);
  const double U = S0 * uf + S1 * vf + S2 * wf;
  const double pf = 0.5 * (R.p + L.p);
  const double rho = 0.5 * (R.rho + L.rho);
  C = rho * U;
  F[0] = C;
  F[1] = C * uf + pf * S0;
  F[2] = C * vf + pf * S1;
  F[3] = C * wf + pf * S2;
  const double Kj = C * 0.5 * (R.u * L.u + R.v * L.v + R.w * L.w);
  const double Pj = 0.5 * (L.p * (R.u * S0 + R.v * S1 + R.w * S2) + R.p * (L.u * S0 + L.v * S1 + L.w * S2));
  const double ef = 2.0 * L.th * R.th / (L.th + R.th) + 0.5 * ((L.e - L.th) + (R.e - R.th));
  F[4] = ef * C + Kj + Pj;
}

// A face side for the Riemann solvers: what hllc, rusanov and ausmup read of
// the reference's FaceState (peregrine/simulator/euler/kernels/flux/recon/constant.mako:3-18
// for a cell as it is, recon/muscl.mako:15-51 for a reconstructed side)
struct RSide {
  double u, v, w, p, rho, e, c;
};

// frompT onto a side (the eos's frompT)
template <int NS, bool RG = false>
__device__ __forceinline__ void side_frompT(const double p, const double T, const double *Y, RSide &s) {
  auto Yf = [&](int n) { return Y[n]; };
  const State th = frompT<NS, decltype(Yf), RG>(p, T, Yf);
  s.p = th.p;
  s.rho = th.rho;
  s.e = th.e;
  s.c = th.c;
}

// b phi(a / b) of the five limiters, b > 0, formed without the ratio
// (peregrine/simulator/euler/kernels/flux/recon/{koren,minmod,mc,superbee,vanleer}.mako);
// the limiter is the case's, the same for every thread
enum { LIM_KOREN = 1, LIM_MINMOD = 2, LIM_MC = 3, LIM_SUPERBEE = 4, LIM_VANLEER = 5 };
__device__ __forceinline__ double bphi(const int lim, const double a, const double b) {
  switch (lim) {
    case LIM_KOREN: return fmax(0.0, fmin(fmin(2.0 * a, (2.0 * b + a) * (1.0 / 3.0)), 2.0 * b));
    case LIM_MINMOD: return fmax(0.0, fmin(b, a));
    case LIM_MC: return fmax(0.0, fmin(fmin(2.0 * a, (b + a) * 0.5), 2.0 * b));
    case LIM_SUPERBEE: return fmax(0.0, fmax(fmin(2.0 * a, b), fmin(a, 2.0 * b)));
    default: return (a + fabs(a)) * b / (b + fabs(a));
  }
}

// the limited slope across a face: the upwind difference dm carried to the
// sign of the difference dp across the face, limited, and the sign put back;
// none where dp is none (recon/muscl.mako:5-13)
__device__ __forceinline__ double phi(const int lim, const double dm, const double dp) {
  double ph = 0.0;
  if (dp != 0.0) {
    const double s = copysign(1.0, dp), a = s * dm, b = fabs(dp);
    ph = s * bphi(lim, a, b);
  }
  return ph;
}
__device__ __forceinline__ double muscl_left(const int lim, const double vLL, const double vL, const double vR) {
  return vL + 0.5 * phi(lim, vL - vLL, vR - vL);
}
__device__ __forceinline__ double muscl_right(const int lim, const double vL, const double vR, const double vRR) {
  return vR - 0.5 * phi(lim, vRR - vR, vR - vL);
}

// HLLC with Davis's outer wave speeds (peregrine/simulator/euler/kernels/flux/function/hllc.mako:2-43)
template <int NS>
__device__ __forceinline__ void hllc(const RSide &L, const RSide &R, const double *YL, const double *YR,
                                     const double *S, double *F) {
  const double area = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
  const double nx = S[0] / area, ny = S[1] / area, nz = S[2] / area;
  const double unL = (L.u * S[0] + L.v * S[1] + L.w * S[2]) / area;
  const double unR = (R.u * S[0] + R.v * S[1] + R.w * S[2]) / area;
  const double SL = unL - L.c, SR = unR + R.c;
  const double Sstar = (R.p - L.p + L.rho * unL * (SL - unL) - R.rho * unR * (SR - unR)) /
                       (L.rho * (SL - unL) - R.rho * (SR - unR));
  bool left, star;
  if (SL >= 0.0) {
    left = true, star = false;
  } else if (Sstar >= 0.0) {
    left = true, star = true;
  } else if (SR >= 0.0) {
    left = false, star = true;
  } else {
    left = false, star = false;
  }
  const RSide &X = left ? L : R;
  const double *Y = left ? YL : YR;
  const double U = left ? unL : unR, SX = left ? SL : SR;
  const double et = X.e + 0.5 * (X.u * X.u + X.v * X.v + X.w * X.w);
  const double mdot = U * X.rho * area;
  F[0] = mdot;
  F[1] = mdot * X.u + X.p * S[0];
  F[2] = mdot * X.v + X.p * S[1];
  F[3] = mdot * X.w + X.p * S[2];
  F[4] = mdot * et + U * X.p * area;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) F[5 + n] = mdot * Y[n];
  if (star) {
    const double rhostar = X.rho * ((SX - U) / (SX - Sstar));
    const double drho = rhostar - X.rho, dU = rhostar * (Sstar - U);
    const double jump = SX * area;
    F[0] += jump * drho;
    F[1] += jump * (drho * X.u + dU * nx);
    F[2] += jump * (drho * X.v + dU * ny);
    F[3] += jump * (drho * X.w + dU * nz);
    F[4] += jump * (drho * et + dU * (Sstar + X.p / (X.rho * (SX - U))));
#pragma unroll
    for (int n = 0; n < NS - 1; n++) F[5 + n] += jump * drho * Y[n];
  }
}

// Rusanov with Davis's bound on the fastest wave
// (peregrine/simulator/euler/kernels/flux/function/rusanov.mako:2-21)
template <int NS>
__device__ __forceinline__ void rusanov(const RSide &L, const RSide &R, const double *YL, const double *YR,
                                        const double *S, double *F) {
  const double area = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
  const double unL = (L.u * S[0] + L.v * S[1] + L.w * S[2]) / area;
  const double unR = (R.u * S[0] + R.v * S[1] + R.w * S[2]) / area;
  const double lam = fmax(fabs(unL) + L.c, fabs(unR) + R.c) * area;
  const double UL = unL * area, UR = unR * area;
  F[0] = 0.5 * (UR * R.rho + UL * L.rho - lam * (R.rho - L.rho));
  F[1] = 0.5 * (UR * R.rho * R.u + R.p * S[0] + UL * L.rho * L.u + L.p * S[0] - lam * (R.rho * R.u - L.rho * L.u));
  F[2] = 0.5 * (UR * R.rho * R.v + R.p * S[1] + UL * L.rho * L.v + L.p * S[1] - lam * (R.rho * R.v - L.rho * L.v));
  F[3] = 0.5 * (UR * R.rho * R.w + R.p * S[2] + UL * L.rho * L.w + L.p * S[2] - lam * (R.rho * R.w - L.rho * L.w));
  const double EL = L.rho * (L.e + 0.5 * (L.u * L.u + L.v * L.v + L.w * L.w));
  const double ER = R.rho * (R.e + 0.5 * (R.u * R.u + R.v * R.v + R.w * R.w));
  F[4] = 0.5 * (UR * (ER + R.p) + UL * (EL + L.p) - lam * (ER - EL));
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double rhoYL = L.rho * YL[n], rhoYR = R.rho * YR[n];
    F[5 + n] = 0.5 * (rhoYR * UR + rhoYL * UL - lam * (rhoYR - rhoYL));
  }
}

// AUSM+-up of Liou (2006) with the cut-off Mach number sqrt(0.1)
// (peregrine/simulator/euler/kernels/flux/function/ausmup.mako:2-38)
template <int NS>
__device__ __forceinline__ void ausmup(const RSide &L, const RSide &R, const double *YL, const double *YR,
                                       const double *S, double *F) {
  const double area = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]), invarea = 1.0 / area;
  const double UL = (L.u * S[0] + L.v * S[1] + L.w * S[2]) * invarea;
  const double UR = (R.u * S[0] + R.v * S[1] + R.w * S[2]) * invarea;
  const double a12 = 0.5 * (R.c + L.c), inva12 = 1.0 / a12;
  const double ML = UL * inva12, MR = UR * inva12;
  const double Mbarsq = 0.5 * (UL * UL + UR * UR) * inva12 * inva12;
  const double Mco = 0.31622776601683794, Kp = 0.25, Ku = 0.75, sigma = 1.0, beta = 1.0 / 8.0;
  const double Mo = sqrt(fmin(1.0, fmax(Mbarsq, Mco * Mco)));
  const double fa = Mo * (2.0 - Mo);
  const double M1p = 0.5 * (ML + fabs(ML)), M1m = 0.5 * (MR - fabs(MR));
  const double M2pL = 0.25 * (ML + 1.0) * (ML + 1.0), M2mL = -0.25 * (ML - 1.0) * (ML - 1.0);
  const double M2pR = 0.25 * (MR + 1.0) * (MR + 1.0), M2mR = -0.25 * (MR - 1.0) * (MR - 1.0);
  const double M4p = fabs(ML) >= 1.0 ? M1p : M2pL * (1.0 - 16.0 * beta * M2mL);
  const double M4m = fabs(MR) >= 1.0 ? M1m : M2mR * (1.0 + 16.0 * beta * M2pR);
  const double alpha = 3.0 / 16.0 * (-4.0 + 5.0 * fa * fa);
  const double p5p = fabs(ML) >= 1.0 ? (ML > 0.0 ? 1.0 : 0.0) : M2pL * ((2.0 - ML) - 16.0 * alpha * ML * M2mL);
  const double p5m = fabs(MR) >= 1.0 ? (MR < 0.0 ? 1.0 : 0.0) : M2mR * ((-2.0 - MR) + 16.0 * alpha * MR * M2pR);
  const double rho12 = 0.5 * (R.rho + L.rho);
  const double M12 = M4p + M4m - Kp * fmax(1.0 - sigma * Mbarsq, 0.0) * (R.p - L.p) * inva12 * inva12 / (fa * rho12);
  const double mdot = a12 * M12 * (M12 > 0.0 ? L.rho : R.rho) * area;
  const double p12 = p5p * L.p + p5m * R.p - Ku * p5p * p5m * (R.rho + L.rho) * fa * a12 * (UR - UL);
  const bool left = mdot > 0.0;
  const RSide &U = left ? L : R;
  const double *Y = left ? YL : YR;
  F[0] = mdot;
  F[1] = mdot * U.u + p12 * S[0];
  F[2] = mdot * U.v + p12 * S[1];
  F[3] = mdot * U.w + p12 * S[2];
  F[4] = mdot * (U.e + 0.5 * (U.u * U.u + U.v * U.v + U.w * U.w) + U.p / U.rho);
#pragma unroll
  for (int n = 0; n < NS - 1; n++) F[5 + n] = mdot * Y[n];
}

enum { FN_HLLC = 1, FN_RUSANOV = 2, FN_AUSMUP = 3 };
template <int FN, int NS>
__device__ __forceinline__ void riemann(const RSide &L, const RSide &R, const double *YL, const double *YR,
                                        const double *S, double *F) {
  if (FN == FN_HLLC) hllc<NS>(L, R, YL, YR, S, F);
  else if (FN == FN_RUSANOV) rusanov<NS>(L, R, YL, YR, S, F);
  else ausmup<NS>(L, R, YL, YR, S, F);
}

// What alpha damping reads of a face's geometry, formed once per face
// (peregrine/simulator/navstokes/kernels/flux/alpha-damping.mako:13-27)
struct FaceGeom {
  double S0, S1, S2;           // area vector
  double dampx, dampy, dampz;  // alpha / |e.n| along the unit normal
  double xLx, xLy, xLz, xRx, xRy, xRz;  // face centre less each cell centre
};

__device__ __forceinline__ FaceGeom face_geom(const double S0, const double S1, const double S2,
                                              const double *xf, const double *xL, const double *xR) {
  FaceGeom g;
  g.S0 = S0, g.S1 = S1, g.S2 = S2;
  const double Sabs = sqrt(S0 * S0 + S1 * S1 + S2 * S2), Sinv = 1.0 / Sabs;
  const double nx = S0 * Sinv, ny = S1 * Sinv, nz = S2 * Sinv;
  const double ex = xR[0] - xL[0], ey = xR[1] - xL[1], ez = xR[2] - xL[2];
  const double en0 = ex * nx, en1 = ey * ny, en2 = ez * nz;
  const double dampinv = kSp.alpha / sqrt(en0 * en0 + en1 * en1 + en2 * en2);
  g.dampx = dampinv * nx, g.dampy = dampinv * ny, g.dampz = dampinv * nz;
  g.xLx = xf[0] - xL[0], g.xLy = xf[1] - xL[1], g.xLz = xf[2] - xL[2];
  g.xRx = xf[0] - xR[0], g.xRy = xf[1] - xR[1], g.xRz = xf[2] - xR[2];
  return g;
}

// the face gradient of one row (alpha-damping.mako:29-38)
__device__ __forceinline__ void facegrad(const FaceGeom &g, const double phiL, const double phiR,
                                         const double *gL, const double *gR, double &gx, double &gy,
                                         double &gz) {
  const double wl = phiL + gL[0] * g.xLx + gL[1] * g.xLy + gL[2] * g.xLz;
  const double wr = phiR + gR[0] * g.xRx + gR[1] * g.xRy + gR[2] * g.xRz;
  const double jump = wr - wl;
  gx = 0.5 * (gR[0] + gL[0]) + g.dampx * jump;
  gy = 0.5 * (gR[1] + gL[1]) + g.dampy * jump;
  gz = 0.5 * (gR[2] + gL[2]) + g.dampz * jump;
}

// The viscous rows of a single-species face (alpha-damping.mako:39-58 and
// :92): with one species every diffusion term of :59-91 is zero, so the
// energy row is the stress work plus the heat flux.  Gradient rows are
// u, v, w, T, each 3 wide.
__device__ __forceinline__ void viscous1(const FaceGeom &g, const double mu, const double kappa,
                                         const double uL, const double vL, const double wL,
                                         const double TL, const double uR, const double vR,
                                         const double wR, const double TR, const double *gL,
                                         const double *gR, double *F) {
  const double lambda = 0.0 - 2.0 / 3.0 * mu;
  double dudx, dudy, dudz, dvdx, dvdy, dvdz, dwdx, dwdy, dwdz;
  facegrad(g, uL, uR, gL + 0, gR + 0, dudx, dudy, dudz);
  facegrad(g, vL, vR, gL + 3, gR + 3, dvdx, dvdy, dvdz);
  facegrad(g, wL, wR, gL + 6, gR + 6, dwdx, dwdy, dwdz);
  const double div = dudx + dvdy + dwdz;
  const double txx = -2.0 * mu * dudx - lambda * div;
  const double txy = -mu * (dvdx + dudy);
  const double txz = -mu * (dwdx + dudz);
  const double tyy = -2.0 * mu * dvdy - lambda * div;
  const double tyz = -mu * (dwdy + dvdz);
  const double tzz = -2.0 * mu * dwdz - lambda * div;
  F[1] += txx * g.S0 + txy * g.S1 + txz * g.S2;
  F[2] += txy * g.S0 + tyy * g.S1 + tyz * g.S2;
  F[3] += txz * g.S0 + tyz * g.S1 + tzz * g.S2;
  double dTx, dTy, dTz;
  facegrad(g, TL, TR, gL + 9, gR + 9, dTx, dTy, dTz);
  const double heatflux = -kappa * (dTx * g.S0 + dTy * g.S1 + dTz * g.S2);
  const double uf = 0.5 * (uR + uL), vf = 0.5 * (vR + vL), wf = 0.5 * (wR + wL);
  const double f4 = (uf * txx + vf * txy + wf * txz) * g.S0 + (uf * txy + vf * tyy + wf * tyz) * g.S1 +
                    (uf * txz + vf * tyz + wf * tzz) * g.S2 + heatflux;
  F[4] += f4;
}

}  // namespace pgb

#include "realgas.cuh"
