// TEST INFRASTRUCTURE ONLY: the CPU oracle the parity tests, smoke() and the
// bench's CPU-baseline leg check the device path against.  Nothing in the
// product links, loads or calls it.
//
// A CPU restatement of PEREGRINE's right-hand side and Runge-Kutta stage for
// the calorically perfect gas, in the reference's own structure: separate
// passes over the blocks in the order its slot graphs run them
// (peregrine/simulator/advec/simulator.py:57-87,
//  peregrine/simulator/advecdiff/simulator.py:110-124), each pass the
// reference template's arithmetic in the same operation order.  Every
// function cites the template it follows.  Built with -ffp-contract=off so no
// multiply-add is fused: the arithmetic is IEEE double as numpy's.
//
// Arrays are the reference's host views: numpy C order, [i][j][k][comp...],
// full extents including ng halo layers (peregrine/backend/allocation.py:8-37).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <cfloat>
#include <omp.h>

extern "C" {

enum { O_EULER = 0, O_NAVSTOKES = 1 };
enum { O_KEPAEC = 0, O_HLLC = 1, O_RUSANOV = 2, O_AUSMUP = 3 };

// one boundary face: block, face (1..6, i-low .. k-high), kind (1..12 in the
// order slp-adia-wall, slp-isot-wall, no-slp-adia-wall, mov-adia-wall,
// no-slp-isot-wall, mov-isot-wall, sub-in-fvt, sup-in-fa, sub-in-ftptt,
// sub-in-fmt, sub-out-fp, sup-out-fn) and the entry's values at the face's
// cells, vals[p][q][nval] with p the lower in-plane axis's interior index
// (the caller evaluates the values at the face centres and the stage's time)
struct OBc {
  int blk, nface, kind, nval;
  const double *vals;
};

struct OCase {
  int simulator;   // O_EULER / O_NAVSTOKES
  int primary;     // flux function
  int ns;          // species
  double alpha;    // alpha-damping coefficient (alpha-damping.mako:11)
  // species tables, ns long (wilkepair ns*ns, row-major [n][m])
  const double *Rsp, *cp0, *h298R, *MWinv, *hpoly0, *h298;
  const double *mu0, *kappa0, *MWqinv, *wilkepair, *lewis;
  double Ru;
  int skip_adv;    // 1: the face fluxes hold the diffusive flux alone (a test's view)
  int recon;       // 0 constant, 1 muscl
  int limiter;     // 1 koren, 2 minmod, 3 mc, 4 superbee, 5 vanleer
  int eos;         // 0 calorically perfect, 1 thermally perfect
  int ncp;         // thermally perfect: terms of cppolyR, cp / R_sp in ln T times R_sp
  const double *cppolyR;  // [ns][ncp]
  int nh;          // terms of hpoly (0: the one term hpoly0)
  const double *hpoly;    // [ns][nh]
  int trans;       // 0 constant properties, 1 kinetic theory
  int nmu, nkappa;        // kinetic theory: terms of the fits below
  const double *mupoly, *kappapoly;  // [ns][nmu] sqrt(mu) / T^(1/4), [ns][nkappa] kappa / sqrt(T), in ln T
  const struct OMech *mech;  // finite-rate chemistry, coupled; null for none
  int realgas, df;           // the cubic real gas; its double flux (euler-df)
  double cu, cw, csigma, ceps;
  const double *csqrtac, *cb, *cda, *cmTc, *conepm, *vshift, *csqrtacMW, *cbMW, *cdaMW, *vshiftMW;  // [ns]
  int nbc;                   // boundary faces; a boundary face not listed keeps its halo as set
  const OBc *bc;
  // the chemistry's integration: 0 the coupled source, 1 sub-stepped over dt
  // (simulator/chemint/substepped.py) with its cap, the tolerance of its
  // equilibrium exit, cp / R_sp in ln T [ns][ncppoly], the molar masses and
  // the exit's concentration floor
  int substepped, cap;
  double eqtol, dt;
  int ncppoly;
  const double *cppoly, *MW;
  double cfloor;
  // binary diffusion (simulator/mixture/diffusion/binary.py): the pair fits
  // [ns][width][nfit], the self fits [ns][nfit], and a partial bath's species
  int binary, bwidth, nfit, bpartial;
  const double *pairfit, *selffit;
  const int *bath;
  // the rotational periodics' rotations, 3 x 3 each, a halo entry's rot
  // (1 + its index, 0 for none) naming one
  const double *rots;
  // Herning's viscosity mixing rule (simulator/mixture/mixrule/herning.py), sqrt(MW) per species
  int herning;
  const double *sqrtMW;
};

// one reaction, the columns of FiniteRateModel.rxnconsts
// (simulator/mixture/chemistry/finiterate.py:122-160) with their counts
enum { O_ELEMENTARY = 0, O_THREEBODY = 1, O_LINDEMANN = 2, O_TROE = 3, O_MAXSIDE = 8 };
struct ORxn {
  int kind, reversible, product, tb, troe, nfcent;
  int nfwd, nreact, nprod, nnet;
  int fwdsp[O_MAXSIDE], reactsp[O_MAXSIDE], prodsp[O_MAXSIDE], netsp[O_MAXSIDE];
  double fwdorder[O_MAXSIDE], reactnu[O_MAXSIDE], prodnu[O_MAXSIDE], netnu[O_MAXSIDE], netnuMW[O_MAXSIDE];
  double logA, b, EaR, logprA, prb, prEaR, nusum;
};
// a third-body set: default efficiency and the deviations from it
struct OTb {
  double defeff;
  int neff;
  int effsp[16];
  double effdev[16];
};
struct OMech {
  int nr, ntb, nlfc, ng;
  const ORxn *rxn;
  const OTb *tb;
  const double *lfcpoly;  // [troe rows][nlfc]
  const double *gpoly;    // [ns][ng]: g / Ru T in ln T, less h298 / T
  const double *h298;     // [ns]
  int logform, product;   // whether any reaction takes the log form / the product form
  double logprefRu, prefRu, Rupref, logcfloor, maxgain, troeuc, troeuhinv;
  double expclamp;        // ln(DBL_MAX) - ln(2 maxgain), as the host works it out
  double lfcfloor;        // log10 of the smallest normal double, a centre without terms
};

struct OBlock {
  int nx, ny, nz, ng;                       // interior cells, halo depth
  double *Q;                                // [nx+2g][ny+2g][nz+2g][ne]
  const double *xcc, *detJinv, *Jinv;       // cells: [..][3], [..], [..][3][3]
  const double *S[3], *xf[3];               // faces of axis a: [..][3]
  double *Tg;                               // [..]: each cell's last T, an iterative eos's starting guess
  double *pst;                              // [..][NSTATE]: the double flux's kept state and frozen planes
  int *subs;                                // [..]: the sub-stepped chemistry's count per cell, or null
};

// one halo cell of one block filled from a cell of another (the place kernel,
// peregrine/multiblock/collections/exchange/kernels/place.mako:11-20, on the
// windows peregrine/multiblock/collections/exchange/collection.py:63-96 lays
// out): dst block, dst i j k, src block, src i j k, and the halo layer
// (0 = next to the interface), all full-array indices.
struct OHaloEntry {
  int32_t dblk, di, dj, dk, sblk, si, sj, sk, layer, rot;
};

}  // extern "C"

namespace {

struct Dims {
  int X, Y, Z;  // full extents
  long at(int i, int j, int k) const { return ((long)i * Y + j) * Z + k; }
};

Dims cells(const OBlock &b) { return {b.nx + 2 * b.ng, b.ny + 2 * b.ng, b.nz + 2 * b.ng}; }
Dims face_dims(const OBlock &b, int a) {
  Dims d = cells(b);
  if (a == 0) d.X += 1;
  if (a == 1) d.Y += 1;
  if (a == 2) d.Z += 1;
  return d;
}

// EosState, simulator/mixture/eos/base.py:85-86: p, T, rhoinv, rho, e, cp, gamma, c
struct State {
  double p, T, rhoinv, rho, e, cp, gamma, c;
};
// the per-cell state record: EosState, then the real gas's Z and the double
// flux's plane theta, eps, kappa, zeta[ns - 1]
enum { NSTATE = 24, S_Z = 8, S_THETA = 9, S_EPS = 10, S_KAPPA = 11, S_ZETA = 12 };

// mixmom, simulator/mixture/eos/kernels/mixing.mako:3-30: cpg's moments are
// R <- Rsp, cp <- cp0, h298 <- h298R (simulator/mixture/eos/cpg/__init__.py),
// tpg's R <- Rsp, cpcoeff[m] <- cppolyR[m], h298 <- h298R
// (simulator/mixture/eos/tpg/model.py:7-9)
enum { O_MAXTERMS = 16 };
struct Mom {
  double R, cp, h298;
  double cpcoeff[O_MAXTERMS];
};
template <class YF> Mom mixmom(const OCase &c, YF Y) {
  Mom m{};
  const bool tpg = c.eos == 1;
  double Ylast = 1.0;
  for (int n = 0; n < c.ns - 1; n++) {
    const double Yn = Y(n);
    Ylast -= Yn;
    m.R += Yn * c.Rsp[n];
    if (tpg)
      for (int t = 0; t < c.ncp; t++) m.cpcoeff[t] += Yn * c.cppolyR[n * c.ncp + t];
    else
      m.cp += Yn * c.cp0[n];
    m.h298 += Yn * c.h298R[n];
  }
  const int L = c.ns - 1;
  m.R += Ylast * c.Rsp[L];
  if (tpg)
    for (int t = 0; t < c.ncp; t++) m.cpcoeff[t] += Ylast * c.cppolyR[L * c.ncp + t];
  else
    m.cp += Ylast * c.cp0[L];
  m.h298 += Ylast * c.h298R[L];
  return m;
}

// ideal_cph: cp and h per mass of the moments at T, h's coefficients built
// from cp's in the same descent (simulator/mixture/caloric/tdepcp/kernels/caloric.mako:4-15)
void ideal_cph(const OCase &c, const Mom &mom, double T, double &cp, double &h) {
  const double u = std::log(T);
  cp = 0.0;
  h = 0.0;
  double hcoeff = 0.0;
  for (int m = c.ncp - 1; m >= 0; m--) {
    cp = cp * u + mom.cpcoeff[m];
    hcoeff = mom.cpcoeff[m] - (m + 1) * hcoeff;
    h = h * u + hcoeff;
  }
  h = h * T + mom.h298;
}

// efromQ (simulator/euler/kernels/solution.mako:10-12)
double efromQ(const double *Q, double rhoinv) {
  return (Q[4] - 0.5 * ((Q[1]) * (Q[1]) + (Q[2]) * (Q[2]) + (Q[3]) * (Q[3])) * rhoinv) * rhoinv;
}

// fromQ (simulator/euler/kernels/state/fromQ.mako:5-19) with cpg's fromrhoE
// (simulator/mixture/eos/cpg/kernels/eos.mako:5-15) or tpg's: Newton from the
// cell's last T, 300 K below 1 K, at least three steps and at most twelve,
// stopping once a step is within 1e5 eps of T; cp is left at the T before
// the last step (simulator/mixture/eos/tpg/kernels/eos.mako:8-20,
// simulator/mixture/eos/tpg/kernels/newton.mako:3-10)
State fromQ(const OCase &c, const double *Q, double Tguess = 0.0) {
  const double rho = Q[0], rhoinv = 1.0 / rho;
  const double e = efromQ(Q, rhoinv);
  Mom mom = mixmom(c, [&](int n) { return Q[5 + n] * rhoinv; });
  State s;
  if (c.eos == 1) {
    double T = (Tguess < 1.0) ? 300.0 : Tguess;
    double cp = 0.0, h = 0.0;
    const double tol = 1e5 * DBL_EPSILON;
    for (int k = 0; k < 12; k++) {
      ideal_cph(c, mom, T, cp, h);
      const double dT = (e - (h - mom.R * T)) / (cp - mom.R);
      T += dT;
      if (k >= 2 && std::fabs(dT) <= tol * T) break;
    }
    s.rho = rho;
    s.rhoinv = 1.0 / rho;
    s.e = e;
    s.T = T;
    s.p = rho * mom.R * T;
    s.cp = cp;
    s.gamma = cp / (cp - mom.R);
    s.c = std::sqrt(s.gamma * mom.R * T);
    return s;
  }
  const double cv = mom.cp - mom.R;
  s.rho = rho;
  s.rhoinv = 1.0 / rho;
  s.e = e;
  s.T = (e - mom.h298) / cv;
  s.p = rho * mom.R * s.T;
  s.cp = mom.cp;
  s.gamma = mom.cp / cv;
  s.c = std::sqrt(s.gamma * mom.R * s.T);
  return s;
}

// frompT: cpg (simulator/mixture/eos/cpg/kernels/eos.mako:17-27), tpg
// (simulator/mixture/eos/tpg/kernels/eos.mako:22-32)
// the real gas's frompT and species enthalpies, further down
template <class YF> State rfrompT(const OCase &c, double p, double T, YF Y, double &Zout);
template <class YF> void rhspecies(const OCase &c, double *h, YF Y, double p, double T, double Z);

State frompT(const OCase &c, double p, double T, const double *Y) {
  if (c.realgas) {
    double Z;
    return rfrompT(c, p, T, [&](int n) { return Y[n]; }, Z);
  }
  Mom mom = mixmom(c, [&](int n) { return Y[n]; });
  State s;
  s.p = p;
  s.T = T;
  s.rho = p / (mom.R * T);
  s.rhoinv = 1.0 / s.rho;
  if (c.eos == 1) {
    double cp, h;
    ideal_cph(c, mom, T, cp, h);
    s.e = h - mom.R * T;
    s.cp = cp;
    s.gamma = cp / (cp - mom.R);
  } else {
    const double cv = mom.cp - mom.R;
    s.e = cv * T + mom.h298;
    s.cp = mom.cp;
    s.gamma = mom.cp / cv;
  }
  s.c = std::sqrt(s.gamma * mom.R * T);
  return s;
}

// fromprims (simulator/euler/kernels/state/fromprims.mako:4-12 through
// solution.mako:2-23 and the eos's frompT); returns the stored T
double fromprims(const OCase &c, const double *q, double *Q) {
  const double u[3] = {q[1], q[2], q[3]};
  const State th = frompT(c, q[0], q[4], q + 5);
  Q[0] = th.rho;
  Q[1] = th.rho * u[0];
  Q[2] = th.rho * u[1];
  Q[3] = th.rho * u[2];
  Q[4] = th.rho * (th.e + 0.5 * ((u[0]) * (u[0]) + (u[1]) * (u[1]) + (u[2]) * (u[2])));
  for (int n = 0; n < c.ns - 1; n++) Q[5 + n] = th.rho * q[5 + n];
  return th.T;
}

// transport (simulator/navstokes/kernels/transport.mako:5-35) with constant
// species properties (simulator/mixture/transport/kernels/constant.mako:5-16),
// Wilke's rule (simulator/mixture/mixrule/kernels/wilke.mako:3-17), the
// series/parallel conductivity (simulator/mixture/transport/kernels/mixing.mako:3-10),
// Lewis diffusivities (simulator/mixture/diffusion/kernels/lewis.mako:3-8) and
// the species enthalpies (simulator/mixture/eos/kernels/species.mako:9-36)
void transport(const OCase &c, const double *Q, const State &st, double *tr, double *hsp, double Z = 0.0) {
  const int ns = c.ns;
  const double rho = Q[0], rhoinv = 1.0 / rho;
  double Ylast = 1.0;
  for (int n = 0; n < ns - 1; n++) Ylast -= Q[5 + n] * rhoinv;
  Ylast = std::fmax(Ylast, 0.0);
  auto Y = [&](int n) { return n < ns - 1 ? Q[5 + n] * rhoinv : Ylast; };
  double denom = 0.0;
  for (int n = 0; n < ns; n++) denom += Y(n) * c.MWinv[n];
  const double MWmix = 1.0 / denom;
  auto X = [&](int n) { return Y(n) * c.MWinv[n] * MWmix; };
  const double T = st.T, lnT = std::log(T);
  std::vector<double> sqrtmu(ns), sinv(ns), kappasp(ns);
  // dilute kinetic theory (simulator/mixture/transport/kernels/dilute.mako:5-26)
  // or constant properties (simulator/mixture/transport/kernels/constant.mako:5-16)
  const double sqrtT = std::sqrt(T), sqrtsqrtT = std::sqrt(sqrtT);
  for (int n = 0; n < ns; n++) {
    if (c.trans == 1) {
      double fit = 0.0;
      for (int m = c.nmu - 1; m >= 0; m--) fit = fit * lnT + c.mupoly[n * c.nmu + m];
      sqrtmu[n] = fit * sqrtsqrtT;
    } else {
      sqrtmu[n] = std::sqrt(c.mu0[n]);
    }
  }
  for (int n = 0; n < ns; n++) sinv[n] = 1.0 / (sqrtmu[n] * c.MWqinv[n]);
  double mu = 0.0;
  if (c.herning) {
    // simulator/mixture/mixrule/kernels/herning.mako:3-12
    double num = 0.0, den = 0.0;
    for (int n = 0; n < ns; n++) {
      const double w = X(n) * c.sqrtMW[n];
      num += w * sqrtmu[n] * sqrtmu[n];
      den += w;
    }
    mu = num / den;
  } else {
    for (int n = 0; n < ns; n++) {
      const double sn = sqrtmu[n] * c.MWqinv[n];
      double phi = 0.0;
      for (int m = 0; m < ns; m++) {
        const double r = 1.0 + sn * sinv[m];
        phi += r * r * c.wilkepair[n * ns + m] * X(m);
      }
      mu += sqrtmu[n] * sqrtmu[n] * X(n) / phi;
    }
  }
  for (int n = 0; n < ns; n++) {
    if (c.trans == 1) {
      double fit = 0.0;
      for (int m = c.nkappa - 1; m >= 0; m--) fit = fit * lnT + c.kappapoly[n * c.nkappa + m];
      kappasp[n] = fit * sqrtT;
    } else {
      kappasp[n] = c.kappa0[n];
    }
  }
  double series = 0.0, parallel = 0.0;
  for (int n = 0; n < ns; n++) {
    series += X(n) * kappasp[n];
    parallel += X(n) / kappasp[n];
  }
  const double kappa = 0.5 * (series + 1.0 / parallel);
  tr[0] = mu;
  tr[1] = kappa;
  if (c.binary) {
    // the mixture average of the pair fits (simulator/mixture/diffusion/kernels/binary.mako:13-62)
    const double invT32 = 1.0 / (T * std::sqrt(T));
    const double tiny = 64 * 2.220446049250313e-16;
    for (int n = 0; n < ns; n++) {
      double sum1 = 0.0, sum2 = 0.0, rest = 0.0, bathx = 0.0;
      for (int k = 0; k < c.bwidth; k++) {
        int m;
        double Xm;
        if (c.bpartial) {
          m = c.bath[k];
          Xm = m != n ? std::fmax(X(m), 0.0) : 0.0;
        } else {
          m = k + (k >= n);
          Xm = std::fmax(X(m), 0.0);
        }
        double Dinv = 0.0;
        for (int t = c.nfit - 1; t >= 0; t--) Dinv = Dinv * lnT + c.pairfit[(n * c.bwidth + k) * c.nfit + t];
        Dinv *= invT32 * 1.0;
        sum1 += Xm * Dinv;
        sum2 += Xm * c.MW[m] * Dinv;
        rest += Xm * c.MW[m];
        bathx += Xm;
      }
      double Dinvself = 0.0;
      for (int t = c.nfit - 1; t >= 0; t--) Dinvself = Dinvself * lnT + c.selffit[n * c.nfit + t];
      Dinvself *= invT32 * 1.0;
      const double Xn = std::fmax(X(n), 0.0);
      bool alone;
      double num, den;
      if (c.bpartial) {
        alone = 1.0 - Xn <= tiny || bathx <= tiny;
        num = alone ? 1.0 : rest * bathx;
        den = alone ? st.p * Dinvself : st.p * ((1.0 - Xn) * rest * sum1 + Xn * bathx * sum2);
      } else {
        alone = 1.0 - Xn <= tiny;
        num = alone ? 1.0 : rest;
        den = alone ? st.p * Dinvself : st.p * (rest * sum1 + Xn * sum2);
      }
      tr[2 + n] = (alone || (rest > 0.0 && den > 0.0)) ? num / den : 0.0;
    }
  } else {
    const double kor = kappa * rhoinv / st.cp;
    for (int n = 0; n < ns; n++) tr[2 + n] = kor / c.lewis[n];
  }
  if (c.realgas) {
    rhspecies(c, hsp, [&](int n) { return Q[5 + n] * rhoinv; }, st.p, T, Z);
    return;
  }
  const double u = std::log(T), Tinv = 1.0 / T;
  for (int n = 0; n < ns; n++) {
    double hRT = 0.0;
    if (c.nh > 0)
      for (int m = c.nh - 1; m >= 0; m--) hRT = hRT * u + c.hpoly[n * c.nh + m];
    else
      hRT = hRT * u + c.hpoly0[n];
    hRT += c.h298[n] * Tinv;
    hsp[n] = hRT * T * c.Ru * c.MWinv[n];
  }
}

// tlog and texp: the reference's table log and exp
// (peregrine/backend/base/kernels/mathfns.mako:6-53 on the tables of
// peregrine/backend/base/mathfns.py:1-22): log x as e ln 2 + log m_k + a
// fifth-degree series in u = m / m_k - 1 over 128 mantissa bins; exp x as
// 2^n 2^(j/64) times a sixth-degree series in the remainder.
struct MathTables {
  double logtab[128], rcptab[128], exptab[64];
  MathTables() {
    for (int k = 0; k < 128; k++) {
      const double m = 0.5 + (k + 0.5) / (2 * 128);
      logtab[k] = std::log(m);
      rcptab[k] = 1.0 / m;
    }
    for (int j = 0; j < 64; j++) exptab[j] = std::pow(2.0, j / 64.0);
  }
};
const MathTables &mtab() {
  static const MathTables t;
  return t;
}
const double O_LN2 = 0x1.62e42fefa39efp-1;
const double O_EXPK = 0x1.71547652b82fep+6;          // 64 / ln 2
const double O_LN2BINS_HI = 0x1.62e42fefp-7;          // ln 2 / 64, the head's low 20 bits clear
const double O_LN2BINS_LO = 0x1.473de6af278edp-40;    // the rest

double tlog(double x) {
  const MathTables &t = mtab();
  long long bits;
  std::memcpy(&bits, &x, sizeof bits);
  const int expo = (int)((bits >> 52) & 0x7ff) - 1022;
  const int bin = (int)((bits >> (52 - 7)) & 127);
  bits = (bits & 0x000fffffffffffffLL) | 0x3fe0000000000000LL;
  double mant;
  std::memcpy(&mant, &bits, sizeof mant);
  const double u = mant * t.rcptab[bin] - 1.0;
  double series = 0.2;
  series = series * u - 0.25;
  series = series * u + 1.0 / 3.0;
  series = series * u - 0.5;
  series = series * u + 1.0;
  return expo * O_LN2 + t.logtab[bin] + u * series;
}

double texp(double v) {
  const MathTables &tb = mtab();
  const double t = v * O_EXPK + 6755399441055744.0;
  long long bits;
  std::memcpy(&bits, &t, sizeof bits);
  const int kexp = (int)bits, nexp = kexp >> 6;
  const double kd = t - 6755399441055744.0;
  const double r = (v - kd * O_LN2BINS_HI) - kd * O_LN2BINS_LO;
  double series = 1.0 / 120.0;
  series = series * r + 1.0 / 24.0;
  series = series * r + 1.0 / 6.0;
  series = series * r + 0.5;
  series = series * r + 1.0;
  series = series * r + 1.0;
  const double m = tb.exptab[kexp & 63] * series;
  std::memcpy(&bits, &m, sizeof bits);
  bits += (long long)(nexp > -1022 ? nexp : -1022) << 52;
  double y;
  std::memcpy(&y, &bits, sizeof y);
  return y;
}

// g / Ru T of species n at ln T u: gpoly's Horner plus h298 / T
// (simulator/mixture/eos/kernels/species.mako:17-22)
double gRTspecies(const OMech &m, int n, double u, double Tinv) {
  double g = 0.0;
  for (int t = m.ng - 1; t >= 0; t--) g = g * u + m.gpoly[n * m.ng + t];
  return g + m.h298[n] * Tinv;
}

// a cell's rate state (simulator/mixture/chemistry/kernels/finiterate.mako:136-183)
struct RateState {
  double T, logT, Tinv, logprefRuT, prefRuT, prefRuTinv, ctot;
  double logc[16], gRT[16], cG[16], logtb[16], ctb[16];
};

template <class YF>
void ratestate(const OCase &c, RateState &s, double rho, YF Y, double T) {
  const OMech &m = *c.mech;
  s.T = T;
  s.logT = tlog(T);
  s.Tinv = 1.0 / T;
  if (m.logform) s.logprefRuT = m.logprefRu - s.logT;
  if (m.product) {
    s.prefRuT = m.prefRu * s.Tinv;
    s.prefRuTinv = m.Rupref * T;
  }
  s.ctot = 0.0;
  for (int n = 0; n < c.ns; n++) {
    const double cn = rho * Y(n) * c.MWinv[n];
    s.ctot += cn;
    s.gRT[n] = gRTspecies(m, n, s.logT, s.Tinv);
    if (m.logform) s.logc[n] = std::fmax(m.logcfloor, tlog(cn));
    if (m.product) s.cG[n] = std::fmax(cn, 0.0) * texp(s.gRT[n]);
  }
  for (int j = 0; j < m.ntb; j++) {
    const OTb &tb = m.tb[j];
    double ctbc = tb.defeff * s.ctot;
    for (int i = 0; i < tb.neff; i++) {
      const int sp = tb.effsp[i];
      ctbc += tb.effdev[i] * (rho * Y(sp) * c.MWinv[sp]);
    }
    s.ctb[j] = ctbc;
    s.logtb[j] = tlog(std::fmax(DBL_MIN, ctbc));
  }
}

// Troe's broadening added to ln k (finiterate.mako:48-63)
double troeblend(const OMech &m, const ORxn &r, const RateState &s, double logpr) {
  const double log10e = 0.4342944819032518, ln10 = 2.302585092994046;
  double lfc;
  if (r.nfcent == 0) {
    lfc = m.lfcfloor;
  } else {
    const double tf = (s.logT - m.troeuc) * m.troeuhinv;
    const double *poly = m.lfcpoly + (long)r.troe * m.nlfc;
    lfc = poly[m.nlfc - 1];
    for (int k = m.nlfc - 2; k >= 0; k--) lfc = lfc * tf + poly[k];
  }
  const double C = -0.4 - 0.67 * lfc, N = 0.75 - 1.27 * lfc;
  const double A = logpr * log10e + C, B = N - 0.14 * A, B2 = B * B;
  return lfc * B2 / (B2 + A * A) * ln10;
}

// one reaction's net rate of progress: the product form (finiterate.mako:66-125)
// or the log form (finiterate.mako:7-46 and the double fold, :201-214)
// one reaction's one-way rates (fwd, rev; rev 0 for an irreversible one)
void oneway(const OMech &m, const ORxn &r, const RateState &s, double &fwd, double &rev) {
  double lk = r.logA;
  if (r.b != 0.0) lk += r.b * s.logT;
  if (r.EaR != 0.0) lk -= r.EaR * s.Tinv;
  const bool falloff = r.kind >= O_LINDEMANN, thirdbody = r.kind != O_ELEMENTARY;
  double logpr = 0.0;
  if (falloff) {
    logpr = s.logtb[r.tb] + r.logprA;
    if (r.prb != 0.0) logpr += r.prb * s.logT;
    if (r.prEaR != 0.0) logpr -= r.prEaR * s.Tinv;
  }
  if (r.product) {
    double pfac = 0.0;
    if (falloff) {
      const double pr = texp(std::fmin(logpr, m.expclamp));
      pfac = pr / (1.0 + pr);
    }
    if (r.kind == O_TROE) lk += troeblend(m, r, s, logpr);
    double xk = lk;
    for (int j = 0; j < r.nreact; j++) xk -= r.reactnu[j] * s.gRT[r.reactsp[j]];
    double K = texp(std::fmin(xk, m.expclamp));
    if (thirdbody && !falloff) K *= s.ctb[r.tb];
    if (falloff) K *= pfac;
    fwd = K;
    for (int j = 0; j < r.nreact; j++)
      for (int q = 0; q < (int)r.reactnu[j]; q++) fwd *= s.cG[r.reactsp[j]];
    rev = 0.0;
    if (r.reversible) {
      rev = K;
      const int nu = (int)std::fabs(r.nusum);
      for (int q = 0; q < nu; q++) rev *= r.nusum > 0 ? s.prefRuTinv : s.prefRuT;
      for (int j = 0; j < r.nprod; j++)
        for (int q = 0; q < (int)r.prodnu[j]; q++) rev *= s.cG[r.prodsp[j]];
    }
    return;
  }
  if (thirdbody && !falloff) lk += s.logtb[r.tb];
  if (falloff) lk += std::fmin(logpr, 0.0) - std::log1p(texp(-std::fabs(logpr)));
  if (r.kind == O_TROE) lk += troeblend(m, r, s, logpr);
  double lrp = lk;
  for (int j = 0; j < r.nfwd; j++) lrp += r.fwdorder[j] * s.logc[r.fwdsp[j]];
  fwd = texp(std::fmin(lrp, m.expclamp));
  rev = 0.0;
  if (!r.reversible) return;
  double diff = r.nusum != 0.0 ? r.nusum * s.logprefRuT : 0.0;
  for (int j = 0; j < r.nnet; j++) diff -= r.netnu[j] * (s.gRT[r.netsp[j]] + s.logc[r.netsp[j]]);
  rev = texp(std::fmin(lrp - diff, m.expclamp));
}

// the fold (finiterate.mako:186-236): the net production rates omega and,
// given D, the destruction rates, kg / m^3 / s; one pass over the reactions
void fold(const OCase &c, const RateState &s, double *omega, double *D) {
  const OMech &m = *c.mech;
  for (int n = 0; n < c.ns; n++) omega[n] = 0.0;
  if (D)
    for (int n = 0; n < c.ns; n++) D[n] = 0.0;
  for (int k = 0; k < m.nr; k++) {
    const ORxn &r = m.rxn[k];
    double fwd, rev;
    oneway(m, r, s, fwd, rev);
    const double rp = r.reversible ? fwd - rev : fwd;
    for (int j = 0; j < r.nnet; j++) {
      const double nuMW = r.netnuMW[j];
      omega[r.netsp[j]] += nuMW * rp;
      if (D) D[r.netsp[j]] += (nuMW < 0.0 ? -nuMW : 0.0) * fwd + (nuMW > 0.0 ? nuMW : 0.0) * rev;
    }
  }
}

// production: the net mass production rates, kg / m^3 / s (finiterate.mako:186-231)
void production(const OCase &c, const RateState &s, double *omega) { fold(c, s, omega, nullptr); }

// cellrates: the clipped mass fractions (simulator/euler/kernels/solution.mako:25-38),
// the rate state at the cell's T and the production rates
// (simulator/chemint/kernels/cell.mako:5-12)
void cellrates(const OCase &c, const double *Q, double T, double *omega) {
  const int ns = c.ns;
  const double rhoinv = 1.0 / Q[0];
  double Ylast = 1.0, Ysum = 0.0;
  for (int n = 0; n < ns - 1; n++) {
    const double Yn = std::fmax(std::fmin(Q[5 + n] * rhoinv, 1.0), 0.0);
    Ylast -= Yn;
    Ysum += Yn;
  }
  const double Yscale = 1.0 / std::fmax(Ysum, 1.0);
  Ylast = std::fmax(Ylast, 0.0);
  auto Y = [&](int n) { return n < ns - 1 ? std::fmax(std::fmin(Q[5 + n] * rhoinv, 1.0), 0.0) * Yscale : Ylast; };
  RateState s;
  ratestate(c, s, Q[0], Y, T);
  production(c, s, omega);
}

// ---- the sub-stepped chemistry (simulator/chemint/kernels/substep.mako,
// bulk.mako, stiff.mako): the one-pass form, every cell with the cap, which
// the compacted passes give to the bit ----

// cp / R and the internal energy per mass of species n (simulator/mixture/eos/kernels/species.mako:3-27)
double cpRof(const OCase &c, int n, double u) {
  double cpR = 0.0;
  for (int m = c.ncppoly - 1; m >= 0; m--) cpR = cpR * u + c.cppoly[n * c.ncppoly + m];
  return cpR;
}
double eof(const OCase &c, int n, double T, double u, double Tinv) {
  double hRT = 0.0;
  for (int m = c.nh - 1; m >= 0; m--) hRT = hRT * u + c.hpoly[n * c.nh + m];
  hRT += c.h298[n] * Tinv;
  return (hRT - 1.0) * T * c.Rsp[n];
}

// integrate (substep.mako:4-87) from Y, T over the step; src the mean rate,
// the substeps taken returned
int integrate(const OCase &c, double rho, double rhoinv, double step, double *Y, double &T, double *src,
              double &remaining, int limit, bool exit) {
  const int ns = c.ns;
  const double eps = 2.220446049250313e-16, tiny = 2.2250738585072014e-308, stepinv = 1.0 / step;
  const double stepfrac = 1e-12;
  auto Yof = [&](int n) { return Y[n]; };
  double rate[16], D[16];
  int sub = 0;
  bool early = false;
  for (; sub < limit && remaining > stepfrac; sub++) {
    RateState s;
    ratestate(c, s, rho, Yof, T);
    fold(c, s, rate, exit && c.eqtol > 0.0 && sub == 0 ? D : nullptr);
    double abest = 0.0, bbest = 0.0;
    for (int n = 0; n < ns; n++) {
      const double sign = std::copysign(1.0, rate[n]);
      const double headroom = 0.5 * ((1.0 - sign) * Y[n] + (1.0 + sign) * (1.0 - Y[n]));
      const double a = rho * std::fmax(headroom, eps), b = std::fmax(std::fabs(rate[n]), tiny);
      if (n == 0 || a * bbest < abest * b) {
        abest = a;
        bbest = b;
      }
    }
    const double share = std::fmin(remaining, abest / bbest * stepinv);
    double cv = 0.0, dTdt = 0.0;
    for (int n = 0; n < ns; n++) {
      const double cpR = cpRof(c, n, s.logT);
      const double e = eof(c, n, T, s.logT, s.Tinv);
      cv += (cpR - 1.0) * c.Rsp[n] * Y[n];
      dTdt -= e * rate[n];
    }
    const double cvrhoinv = 1.0 / (cv * rho);
    dTdt *= cvrhoinv;
    if (exit && c.eqtol > 0.0) {
      const double tleft = remaining * step, tleftinv = 1.0 / tleft;
      bool settled = sub == 0 && tleft > 0.0 && std::fabs(dTdt) * tleft < 0.1;
      for (int n = 0; n < ns && settled; n++) settled = std::fabs(rate[n] * rhoinv) * tleft < c.eqtol;
      if (settled) {
        double dT = 0.0;
        for (int n = 0; n < ns; n++) {
          const double rhoden = rho * std::fmax(Y[n], c.cfloor * c.MW[n] * rhoinv);
          const double move = std::fmax((rate[n] * rhoinv) * tleft * rhoden / (rhoden + D[n] * tleft), -Y[n]);
          const double r = move * rho * tleftinv;
          const double e = eof(c, n, T, s.logT, s.Tinv);
          dT -= e * r;
          Y[n] += move;
          src[n] += r * remaining;
        }
        T += dT * cvrhoinv * tleft;
        remaining = 0.0;
        early = true;
        break;
      }
    }
    const double tsub = share * step;
    for (int n = 0; n < ns; n++) {
      Y[n] += (rate[n] * rhoinv) * tsub;
      src[n] += rate[n] * share;
    }
    T += dTdt * tsub;
    remaining -= share;
    if (share <= stepfrac) {
      remaining = 0.0;
      early = true;
      break;
    }
  }
  return early ? sub + 1 : sub;
}

// a cell's sub-stepped source over the step: the clipped mass fractions
// and the cell's T (substep.mako:89-95), the cap, the exit where the
// tolerance is set; the mean rates into omega, the count returned
int substepped(const OCase &c, const double *Q, double T, double *omega) {
  const int ns = c.ns;
  const double rho = Q[0], rhoinv = 1.0 / Q[0];
  double Ylast = 1.0, Ysum = 0.0;
  for (int n = 0; n < ns - 1; n++) {
    const double Yn = std::fmax(std::fmin(Q[5 + n] * rhoinv, 1.0), 0.0);
    Ylast -= Yn;
    Ysum += Yn;
  }
  const double Yscale = 1.0 / std::fmax(Ysum, 1.0);
  Ylast = std::fmax(Ylast, 0.0);
  double Y[16];
  for (int n = 0; n < ns; n++) {
    Y[n] = n < ns - 1 ? std::fmax(std::fmin(Q[5 + n] * rhoinv, 1.0), 0.0) * Yscale : Ylast;
    omega[n] = 0.0;
  }
  double remaining = 1.0;
  return integrate(c, rho, rhoinv, c.dt, Y, T, omega, remaining, c.cap, true);
}

// ---- the cubic real gas (simulator/mixture/eos/realgas/kernels/eos.mako,
// realgas/kernels/newton.mako) and its double flux
// (simulator/mixture/eos/realgasdf/kernels/eos.mako, simulator/eulerdf/kernels/) ----
struct Cubic {
  double MWmix, bm, cm, S1, S2, am, dam, Astar, Bstar, Cstar, invRuT, Z, z1, z2, invslope, dZdT, v, I, logratio, q, qd;
};
struct RMom {
  double R, h298, b, c, da;
  Mom ideal;  // cp's coefficients and h298, for ideal_cph
};

template <class YF> RMom rmixmom(const OCase &c, YF Y) {
  RMom m{};
  m.ideal = mixmom(c, Y);
  m.R = m.ideal.R, m.h298 = m.ideal.h298;
  double Ylast = 1.0;
  for (int n = 0; n < c.ns - 1; n++) {
    const double Yn = Y(n);
    Ylast -= Yn;
    m.b += Yn * c.cbMW[n];
    m.c += Yn * c.vshiftMW[n];
    m.da += Yn * c.cdaMW[n];
  }
  const int L = c.ns - 1;
  m.b += Ylast * c.cbMW[L];
  m.c += Ylast * c.vshiftMW[L];
  m.da += Ylast * c.cdaMW[L];
  return m;
}

void cubicmix(const OCase &c, Cubic &q, const RMom &m) {
  q.MWmix = c.Ru / m.R;
  q.bm = m.b * q.MWmix;
  q.cm = m.c * q.MWmix;
  q.S2 = m.da * q.MWmix;
}

// sqrt(a_n), whole or per unit of Y_n / MW_n, Soave's modulus opened (eos.mako:5-8)
double sqrtaMW(const OCase &c, int n, double sqrtT) {
  return c.csqrtacMW[n] * std::fabs(std::fma(-sqrtT, c.cmTc[n], c.conepm[n]));
}
double sqrta(const OCase &c, int n, double sqrtT) {
  return c.csqrtac[n] * std::fabs(std::fma(-sqrtT, c.cmTc[n], c.conepm[n]));
}

template <class YF> void attraction(const OCase &c, Cubic &q, YF Y, double T) {
  const double sqrtT = std::sqrt(T);
  double s1 = 0.0, Ylast = 1.0;
  for (int n = 0; n < c.ns - 1; n++) {
    const double Yn = Y(n);
    Ylast -= Yn;
    s1 = std::fma(Yn, sqrtaMW(c, n, sqrtT), s1);
  }
  s1 = std::fma(Ylast, sqrtaMW(c, c.ns - 1, sqrtT), s1);
  q.S1 = s1 * q.MWmix;
  q.am = q.S1 * q.S1;
  q.dam = -q.S1 * q.S2 / sqrtT;
}

void dimless(const OCase &c, Cubic &q, double p, double T) {
  q.invRuT = 1.0 / (c.Ru * T);
  const double pRT = p * q.invRuT;
  q.Astar = q.am * pRT * q.invRuT;
  q.Bstar = q.bm * pRT;
  q.Cstar = q.cm * pRT;
  const double B = q.Bstar, B2 = B * B;
  q.z1 = q.Astar + c.cw * B2 - c.cu * B - c.cu * B2;
  q.z2 = -(1.0 + B - c.cu * B);
}

void rootslope(Cubic &q) { q.invslope = 1.0 / (3.0 * q.Z * q.Z + 2.0 * q.Z * q.z2 + q.z1); }

void zsolve(const OCase &c, Cubic &q, double p, double T) {
  dimless(c, q, p, T);
  const double B = q.Bstar, B2 = B * B, z1 = q.z1, z2 = q.z2;
  const double z0 = -(q.Astar * B + c.cw * B2 * (1.0 + B));
  const double Q = (z2 * z2 - 3.0 * z1) * (1.0 / 9.0);
  const double R = (2.0 * z2 * z2 * z2 - 9.0 * z2 * z1 + 27.0 * z0) * (1.0 / 54.0);
  const double M = R * R - Q * Q * Q;
  const double z2o3 = z2 * (1.0 / 3.0);
  if (M > 0.0) {
    const double S = -std::copysign(std::cbrt(std::fabs(R) + std::sqrt(M)), R);
    q.Z = S + Q / S - z2o3;
  } else {
    const double sqQ = std::sqrt(Q), twopio3 = 2.0943951023931954923;
    const double theta3 = std::acos(R / (Q * sqQ)) * (1.0 / 3.0);
    const double roots[3] = {-2.0 * sqQ * std::cos(theta3) - z2o3, -2.0 * sqQ * std::cos(theta3 + twopio3) - z2o3,
                             -2.0 * sqQ * std::cos(theta3 - twopio3) - z2o3};
    double Z = std::fmax(roots[0], std::fmax(roots[1], roots[2]));
    int above = 0;
    for (int k = 0; k < 3; k++) above += roots[k] > B;
    if (above > 1) {
      const double AoBse = q.Astar / (B * (c.csigma - c.ceps));
      double gmin = 0.0;
      bool found = false;
      for (int k = 0; k < 3; k++) {
        const double z = roots[k];
        if (z <= B) continue;
        const double g = z - 1.0 - std::log(z - B) + AoBse * std::log((z + c.ceps * B) / (z + c.csigma * B));
        if (!found || g < gmin) gmin = g, Z = z, found = true;
      }
    }
    q.Z = Z;
  }
  rootslope(q);
}

double dZ(const OCase &c, const Cubic &q, double dA, double dB) {
  const double B = q.Bstar, Z = q.Z, Z2 = Z * Z;
  const double dz0 = -(B * dA + (q.Astar + (2.0 * B + 3.0 * B * B) * c.cw) * dB);
  const double dz1 = dA + (2.0 * B * (c.cw - c.cu) - c.cu) * dB;
  const double dz2 = -(1.0 - c.cu) * dB;
  return -(dz2 * Z2 + dz1 * Z + dz0) * q.invslope;
}

void departures(const OCase &c, double &hdep, double &cpdep, Cubic &q, double T) {
  const double Tinv = c.Ru * q.invRuT;
  const double dlnamdT = q.dam / q.am;
  q.dZdT = dZ(c, q, -2.0 * q.Astar * Tinv * (1.0 - 0.5 * T * dlnamdT), -q.Bstar * Tinv);
  const double x = q.Z / q.Bstar, xm1 = x - 1.0;
  const double D = x * x + c.cu * x + c.cw;
  q.logratio = std::log((x + c.ceps) / (x + c.csigma));
  const double invBmRu = 1.0 / (q.bm * c.Ru);
  const double hres = invBmRu / (c.csigma - c.ceps) * (q.am * Tinv - q.dam) * q.logratio;
  q.qd = q.dam * invBmRu;
  q.q = q.am * invBmRu * Tinv;
  const double num = D - q.qd * xm1;
  cpdep = hres * 0.5 * T * dlnamdT + num * num / (D * D - q.q * (2.0 * x + c.cu) * xm1 * xm1) - 1.0;
  hdep = hres + (q.Z - 1.0) - q.Cstar;
}

void gamma_c(const OCase &c, double &gamma, double &cs, const Cubic &q, double p, double T, double rho, double cp,
             double invZt) {
  const double invp = 1.0 / p, Tinv = c.Ru * q.invRuT;
  const double dZtdT = q.dZdT + q.Cstar * Tinv;
  const double dZdp = dZ(c, q, q.Astar * invp, q.Bstar * invp);
  const double dZtdp = dZdp - q.Cstar * invp;
  const double drhodp = rho * invp * (1.0 - p * dZtdp * invZt);
  const double r = -Tinv * (1.0 + T * dZtdT * invZt);
  const double csq = 1.0 / (drhodp - (T / cp) * r * r);
  gamma = drhodp * csq;
  cs = std::sqrt(std::fabs(csq));
}

// frompT (eos.mako:139-155); Z out
template <class YF> State rfrompT(const OCase &c, double p, double T, YF Y, double &Zout) {
  const RMom m = rmixmom(c, Y);
  Cubic q{};
  cubicmix(c, q, m);
  attraction(c, q, Y, T);
  double cpi, hi;
  ideal_cph(c, m.ideal, T, cpi, hi);
  zsolve(c, q, p, T);
  double hdep, cpdep;
  departures(c, hdep, cpdep, q, T);
  State s;
  s.p = p;
  s.T = T;
  Zout = q.Z;
  s.cp = cpi + m.R * cpdep;
  const double Zt = q.Z - q.Cstar, invZt = 1.0 / Zt, porho = Zt * m.R * T;
  s.rho = p * q.invRuT * q.MWmix * invZt;
  s.rhoinv = 1.0 / s.rho;
  s.e = hi + m.R * T * hdep - porho;
  gamma_c(c, s.gamma, s.c, q, p, T, s.rho, s.cp, invZt);
  return s;
}

void atvolume(const OCase &c, Cubic &q, double rho) {
  q.v = q.MWmix / rho + q.cm;
  q.I = std::log((q.v + c.csigma * q.bm) / (q.v + c.ceps * q.bm)) / ((c.csigma - c.ceps) * q.bm);
}

// fromrhoE (eos.mako:162-190, realgas/kernels/newton.mako:3-14)
template <class YF> State rfromrhoE(const OCase &c, YF Y, double rho, double e, double Tguess, double &Zout) {
  const RMom m = rmixmom(c, Y);
  Cubic q{};
  cubicmix(c, q, m);
  atvolume(c, q, rho);
  const double invMWmix = 1.0 / q.MWmix;
  double T = (Tguess < 1.0) ? 300.0 : Tguess;
  double cpi = 0.0, hi = 0.0;
  const double tol = 1e5 * DBL_EPSILON;
  for (int k = 0; k < 12; k++) {
    attraction(c, q, Y, T);
    ideal_cph(c, m.ideal, T, cpi, hi);
    const double app = 0.5 * (q.S2 * q.S2 - q.dam) / T;
    const double f = hi - m.R * T - (q.am - T * q.dam) * q.I * invMWmix - e;
    const double cv = cpi - m.R + T * app * q.I * invMWmix;
    const double dT = f / cv;
    T -= dT;
    if (k >= 2 && std::fabs(dT) <= tol * T) break;
  }
  attraction(c, q, Y, T);
  ideal_cph(c, m.ideal, T, cpi, hi);
  const double vs = q.v + c.csigma * q.bm, ve = q.v + c.ceps * q.bm;
  const double p = c.Ru * T / (q.v - q.bm) - q.am / (vs * ve);
  dimless(c, q, p, T);
  q.Z = p * q.invRuT * q.v;
  rootslope(q);
  double hdep, cpdep;
  departures(c, hdep, cpdep, q, T);
  State s;
  s.rho = rho;
  s.rhoinv = 1.0 / rho;
  s.e = e;
  s.p = p;
  s.T = T;
  Zout = q.Z;
  s.cp = cpi + m.R * cpdep;
  const double invZt = 1.0 / (q.Z - q.Cstar);
  gamma_c(c, s.gamma, s.c, q, p, T, rho, s.cp, invZt);
  return s;
}

// fromrhop (realgasdf/kernels/eos.mako:6-30, realgasdf/kernels/newton.mako:3-13)
template <class YF> State rfromrhop(const OCase &c, YF Y, double rho, double p, double Tguess, double &Zout) {
  const RMom m = rmixmom(c, Y);
  Cubic q{};
  cubicmix(c, q, m);
  atvolume(c, q, rho);
  const double vs = q.v + c.csigma * q.bm, ve = q.v + c.ceps * q.bm;
  const double invvmb = 1.0 / (q.v - q.bm), invD = 1.0 / (vs * ve);
  double T = (Tguess < 1.0) ? 300.0 : Tguess;
  const double tol = 1e5 * DBL_EPSILON;
  for (int k = 0; k < 12; k++) {
    attraction(c, q, Y, T);
    const double f = c.Ru * T * invvmb - q.am * invD - p;
    const double dpdT = c.Ru * invvmb - q.dam * invD;
    const double dT = f / dpdT;
    T -= dT;
    if (k >= 2 && std::fabs(dT) <= tol * T) break;
  }
  attraction(c, q, Y, T);
  double cpi, hi;
  ideal_cph(c, m.ideal, T, cpi, hi);
  dimless(c, q, p, T);
  q.Z = p * q.invRuT * q.v;
  rootslope(q);
  double hdep, cpdep;
  departures(c, hdep, cpdep, q, T);
  State s;
  s.rho = rho;
  s.rhoinv = 1.0 / rho;
  s.p = p;
  s.T = T;
  Zout = q.Z;
  s.cp = cpi + m.R * cpdep;
  s.e = hi + m.R * T * hdep - p / rho;
  const double invZt = 1.0 / (q.Z - q.Cstar);
  gamma_c(c, s.gamma, s.c, q, p, T, rho, s.cp, invZt);
  return s;
}

// hspecies at a stored state: hpartialpoint and hpartial (eos.mako:192-224, 257-273)
template <class YF> void rhspecies(const OCase &c, double *h, YF Y, double p, double T, double Z) {
  const RMom m = rmixmom(c, Y);
  Cubic q{};
  cubicmix(c, q, m);
  attraction(c, q, Y, T);
  dimless(c, q, p, T);
  q.Z = Z;
  rootslope(q);
  double hdep, cpdep;
  departures(c, hdep, cpdep, q, T);
  const double lnT = std::log(T), Tinv = c.Ru * q.invRuT, sqrtT = std::sqrt(T);
  const double B = q.Bstar, ZT = q.dZdT, BT = -B * Tinv;
  const double invZsB = 1.0 / (Z + c.csigma * B), invZeB = 1.0 / (Z + c.ceps * B);
  const double Iz = -q.logratio / (c.csigma - c.ceps);
  const double IzT = ((ZT + c.csigma * BT) * invZsB - (ZT + c.ceps * BT) * invZeB) / (c.csigma - c.ceps);
  const double dlnZmB = (ZT - BT) / (Z - B);
  const double invS1 = 1.0 / q.S1, invBm = 1.0 / q.bm;
  const double invamsqrtT = invS1 * invS1 / sqrtT;
  for (int n = 0; n < c.ns; n++) {
    double hRT = 0.0;
    for (int t = c.nh - 1; t >= 0; t--) hRT = hRT * lnT + c.hpoly[n * c.nh + t];
    hRT += c.h298[n] * Tinv;
    const double qT = (q.qd - q.q) * Tinv;
    const double sqrtan = sqrta(c, n, sqrtT);
    const double r = 2.0 * sqrtan * invS1;
    const double rT = (sqrtan * q.S2 - c.cda[n] * q.S1) * invamsqrtT;
    const double bb = c.cb[n] * invBm;
    const double qbar = q.q * (r - bb), qbarT = qT * (r - bb) + q.q * rT;
    const double dlnphidT = bb * q.dZdT - dlnZmB - qbarT * Iz - qbar * IzT;
    h[n] = (hRT * T * c.Ru - c.Ru * T * T * dlnphidT - c.vshift[n] * p) * c.MWinv[n];
  }
}

// drho (eos.mako:226-255)
template <class YF>
void rdrho(const OCase &c, double &rho_p, double &rho_T, double *rho_Y, YF Y, double p, double T, double rho) {
  const RMom m = rmixmom(c, Y);
  Cubic q{};
  cubicmix(c, q, m);
  attraction(c, q, Y, T);
  zsolve(c, q, p, T);
  double hdep, cpdep;
  departures(c, hdep, cpdep, q, T);
  const double invp = 1.0 / p, Tinv = c.Ru * q.invRuT, sqrtT = std::sqrt(T);
  const double Zt = q.Z - q.Cstar, dZtdT = q.dZdT + q.Cstar * Tinv, invZt = 1.0 / Zt;
  const double dZdp = dZ(c, q, q.Astar * invp, q.Bstar * invp);
  rho_p = rho * invp * (1.0 - (p * dZdp - q.Cstar) * invZt);
  rho_T = -rho * Tinv * (1.0 + T * dZtdT * invZt);
  const double twoS1 = 2.0 * q.S1;
  const double invRuT = Tinv / c.Ru, pRT = p * invRuT;
  const int L = c.ns - 1;
  const double MWinv_last = c.MWinv[L], sqrta_last = sqrtaMW(c, L, sqrtT);
  const double b_last = c.cbMW[L], c_last = c.vshiftMW[L];
  for (int n = 0; n < c.ns - 1; n++) {
    const double dlnMWmix = -q.MWmix * (c.MWinv[n] - MWinv_last);
    const double dam = twoS1 * (q.S1 * dlnMWmix + q.MWmix * (sqrtaMW(c, n, sqrtT) - sqrta_last));
    const double dbm = q.bm * dlnMWmix + q.MWmix * (c.cbMW[n] - b_last);
    const double dcm = q.cm * dlnMWmix + q.MWmix * (c.vshiftMW[n] - c_last);
    const double dZdY = dZ(c, q, dam * pRT * invRuT, dbm * pRT);
    rho_Y[n] = rho * (dlnMWmix - (dZdY - dcm * pRT) * invZt);
  }
}

// planeslopes (realgasdf/kernels/eos.mako:32-48)
template <class YF>
void planeslopes(const OCase &c, double &theta, double &epsY, YF Y, double rho, double rhoinv, double T, double e) {
  const RMom m = rmixmom(c, Y);
  Cubic q{};
  cubicmix(c, q, m);
  atvolume(c, q, rho);
  attraction(c, q, Y, T);
  const double vs = q.v + c.csigma * q.bm, ve = q.v + c.ceps * q.bm;
  const double invvmb = 1.0 / (q.v - q.bm), invD = 1.0 / (vs * ve), invMWmix = 1.0 / q.MWmix;
  double cpi, hi;
  ideal_cph(c, m.ideal, T, cpi, hi);
  const double app = 0.5 * (q.S2 * q.S2 - q.dam) / T;
  const double cv = cpi - m.R + T * app * q.I * invMWmix;
  const double p = c.Ru * T * invvmb - q.am * invD;
  const double dpdT = c.Ru * invvmb - q.dam * invD;
  const double dpdrho = q.MWmix * rhoinv * rhoinv * (c.Ru * T * invvmb * invvmb - q.am * (vs + ve) * invD * invD);
  theta = rho * cv / dpdT;
  epsY = e - (T * dpdT - p) * rhoinv - theta * dpdrho;
}

// freeze of one cell: the energy reset to the eos's and the tangent plane
// (simulator/eulerdf/kernels/freeze.mako:3-32); st is the cell's record
void freeze(const OCase &c, double *Q, double *st) {
  const double rho = Q[0], rhoinv = 1.0 / rho;
  const double p = st[0], T = st[1], e = st[4];
  const double rhoe = rho * e;
  Q[4] = rhoe + 0.5 * ((Q[1]) * (Q[1]) + (Q[2]) * (Q[2]) + (Q[3]) * (Q[3])) * rhoinv;
  auto Y = [&](int n) { return Q[5 + n] * rhoinv; };
  double theta, epsY;
  planeslopes(c, theta, epsY, Y, rho, rhoinv, T, e);
  double rho_p, rho_T, rho_Y[16];
  rdrho(c, rho_p, rho_T, rho_Y, Y, p, T, rho);
  double h[16];
  rhspecies(c, h, Y, p, T, st[S_Z]);
  const double cpoverrhoT = st[5] / rho_T;
  double zetaY = 0.0;
  for (int n = 0; n < c.ns - 1; n++) {
    st[S_ZETA + n] = h[n] - h[c.ns - 1] - cpoverrhoT * rho_Y[n];
    zetaY += st[S_ZETA + n] * Y(n);
  }
  st[S_THETA] = theta;
  st[S_EPS] = epsY - zetaY;
  st[S_KAPPA] = rhoe - epsY * rho - theta * p;
}

// the state of one cell from Q: the real gas's fromrhoE, or with plane its
// fromplane, p off the cell's frozen plane (simulator/eulerdf/kernels/fromplane.mako:3-17)
void rstate(const OCase &c, const double *Q, double *st, double Tguess, bool plane) {
  const double rho = Q[0], rhoinv = 1.0 / rho;
  auto Y = [&](int n) { return Q[5 + n] * rhoinv; };
  double Z = 0.0;
  State s;
  if (plane) {
    double composition = 0.0;
    for (int n = 0; n < c.ns - 1; n++) composition += st[S_ZETA + n] * Q[5 + n];
    const double p = (Q[4] - 0.5 * ((Q[1]) * (Q[1]) + (Q[2]) * (Q[2]) + (Q[3]) * (Q[3])) * rhoinv - st[S_EPS] * Q[0] -
                      composition - st[S_KAPPA]) / st[S_THETA];
    s = rfromrhop(c, Y, rho, p, Tguess, Z);
  } else {
    s = rfromrhoE(c, Y, rho, efromQ(Q, rhoinv), Tguess, Z);
  }
  std::memcpy(st, &s, sizeof(State));
  st[S_Z] = Z;
}

// the double flux's kepaec with its two energy rows (eulerdf/kernels/flux/function/kepaec.mako:1-21)
void kepaec_df(const OCase &c, const double *QL, const double *QR, const double *sL, const double *sR,
               const double *S, double *F) {
  const int ns = c.ns, ne = 4 + ns;
  const double uL = QL[1] / QL[0], vL = QL[2] / QL[0], wL = QL[3] / QL[0];
  const double uR = QR[1] / QR[0], vR = QR[2] / QR[0], wR = QR[3] / QR[0];
  const double pL = sL[0], pR = sR[0], rL = sL[3], rR = sR[3];
  const double uf = 0.5 * (uR + uL), vf = 0.5 * (vR + vL), wf = 0.5 * (wR + wL);
  const double U = (S[0]) * (uf) + (S[1]) * (vf) + (S[2]) * (wf);
  const double pf = 0.5 * (pR + pL), rho = 0.5 * (rR + rL);
  const double C = rho * U;
  F[0] = C;
  F[1] = C * uf + pf * S[0];
  F[2] = C * vf + pf * S[1];
  F[3] = C * wf + pf * S[2];
  const double Kj = C * 0.5 * ((uR) * (uL) + (vR) * (vL) + (wR) * (wL));
  const double Pj = 0.5 * (pL * ((uR) * (S[0]) + (vR) * (S[1]) + (wR) * (S[2])) +
                           pR * ((uL) * (S[0]) + (vL) * (S[1]) + (wL) * (S[2])));
  double YL[16], YR[16];
  for (int n = 0; n < ns - 1; n++) {
    YL[n] = QL[5 + n] / QL[0], YR[n] = QR[5 + n] / QR[0];
    F[5 + n] = 0.5 * (YR[n] + YL[n]) * C;
  }
  const double rhoinvL = 1.0 / rL, rhoinvR = 1.0 / rR;
  double cL[2] = {0.0, 0.0}, cR[2] = {0.0, 0.0};
  for (int n = 0; n < ns - 1; n++) {
    cL[0] += sL[S_ZETA + n] * YL[n], cL[1] += sR[S_ZETA + n] * YL[n];
    cR[0] += sL[S_ZETA + n] * YR[n], cR[1] += sR[S_ZETA + n] * YR[n];
  }
  for (int q = 0; q < 2; q++) {
    const double *pl = q == 0 ? sL : sR;
    const double tL = (pl[S_THETA] * pL + pl[S_KAPPA]) * rhoinvL, tR = (pl[S_THETA] * pR + pl[S_KAPPA]) * rhoinvR;
    F[q == 0 ? 4 : ne] = (pl[S_EPS] + 0.5 * (cL[q] + cR[q]) + 2.0 * tL * tR / (tL + tR)) * C + Kj + Pj;
  }
}

// a face's side: the cell's state plus its velocity as Q[1..3] / Q[0]
// (simulator/euler/kernels/flux/recon/constant.mako:3-18)
struct Side {
  State s;
  double u, v, w;
};
Side side(const double *Q, const State &st) {
  return Side{st, Q[1] / Q[0], Q[2] / Q[0], Q[3] / Q[0]};
}

// kepaec (simulator/euler/kernels/flux/function/kepaec.mako:2-20)
void kepaec(const OCase &c, const Side &L, const Side &R, const double *QL, const double *QR,
            const double *S, double *F) {
  const double uf = 0.5 * (R.u + L.u), vf = 0.5 * (R.v + L.v), wf = 0.5 * (R.w + L.w);
  const double U = ((S[0]) * (uf) + (S[1]) * (vf) + (S[2]) * (wf));
  const double pf = 0.5 * (R.s.p + L.s.p);
  const double rho = 0.5 * (R.s.rho + L.s.rho);
  const double C = rho * U;
  F[0] = C;
  F[1] = C * uf + pf * S[0];
  F[2] = C * vf + pf * S[1];
  F[3] = C * wf + pf * S[2];
  const double Kj = C * 0.5 * ((R.u) * (L.u) + (R.v) * (L.v) + (R.w) * (L.w));
  const double Pj = 0.5 * (L.s.p * ((R.u) * (S[0]) + (R.v) * (S[1]) + (R.w) * (S[2])) +
                           R.s.p * ((L.u) * (S[0]) + (L.v) * (S[1]) + (L.w) * (S[2])));
  const double thL = L.s.cp / L.s.gamma * L.s.T, thR = R.s.cp / R.s.gamma * R.s.T;
  const double ef = 2.0 * thL * thR / (thL + thR) + 0.5 * ((L.s.e - thL) + (R.s.e - thR));
  F[4] = ef * C + Kj + Pj;
  for (int n = 0; n < c.ns - 1; n++) F[5 + n] = 0.5 * (QR[5 + n] / QR[0] + QL[5 + n] / QL[0]) * C;
}

// b phi(a / b) of the limiters, b > 0 (simulator/euler/kernels/flux/recon/{koren,minmod,mc,superbee,vanleer}.mako)
double limiter(int which, double a, double b) {
  switch (which) {
    case 1: return std::fmax(0.0, std::fmin(std::fmin(2.0 * a, (2.0 * b + a) * (1.0 / 3.0)), 2.0 * b));
    case 2: return std::fmax(0.0, std::fmin(b, a));
    case 3: return std::fmax(0.0, std::fmin(std::fmin(2.0 * a, (b + a) * 0.5), 2.0 * b));
    case 4: return std::fmax(0.0, std::fmax(std::fmin(2.0 * a, b), std::fmin(a, 2.0 * b)));
    default: return (a + std::fabs(a)) * b / (b + std::fabs(a));
  }
}

// the limited slope across a face (simulator/euler/kernels/flux/recon/muscl.mako:5-13)
double phi(int which, double dm, double dp) {
  double ph = 0.0;
  if (dp != 0.0) {
    const double s = std::copysign(1.0, dp), a = s * dm, b = std::fabs(dp);
    ph = s * limiter(which, a, b);
  }
  return ph;
}

// MUSCL sides (simulator/euler/kernels/flux/recon/muscl.mako:15-51): p, T, Y
// and the velocity limited, each side's state from its p, T, Y by frompT
void muscl(const OCase &c, const double *QLL, const double *QL, const double *QR, const double *QRR,
           const State &sLL, const State &sL, const State &sR, const State &sRR, Side &L, Side &R,
           double *YL, double *YR) {
  const int lim = c.limiter, ns = c.ns;
  auto left = [&](double vLL, double vL, double vR) { return vL + 0.5 * phi(lim, vL - vLL, vR - vL); };
  auto right = [&](double vL, double vR, double vRR) { return vR - 0.5 * phi(lim, vRR - vR, vR - vL); };
  const double riLL = sLL.rhoinv, riL = sL.rhoinv, riR = sR.rhoinv, riRR = sRR.rhoinv;
  const double pL = left(sLL.p, sL.p, sR.p), pR = right(sL.p, sR.p, sRR.p);
  const double TL = left(sLL.T, sL.T, sR.T), TR = right(sL.T, sR.T, sRR.T);
  for (int n = 0; n < ns - 1; n++) {
    YL[n] = left(QLL[5 + n] * riLL, QL[5 + n] * riL, QR[5 + n] * riR);
    YR[n] = right(QL[5 + n] * riL, QR[5 + n] * riR, QRR[5 + n] * riRR);
  }
  L.s = frompT(c, pL, TL, YL);
  L.u = left(QLL[1] * riLL, QL[1] * riL, QR[1] * riR);
  L.v = left(QLL[2] * riLL, QL[2] * riL, QR[2] * riR);
  L.w = left(QLL[3] * riLL, QL[3] * riL, QR[3] * riR);
  R.s = frompT(c, pR, TR, YR);
  R.u = right(QL[1] * riL, QR[1] * riR, QRR[1] * riRR);
  R.v = right(QL[2] * riL, QR[2] * riR, QRR[2] * riRR);
  R.w = right(QL[3] * riL, QR[3] * riR, QRR[3] * riRR);
}

// HLLC with Davis's outer wave speeds (simulator/euler/kernels/flux/function/hllc.mako:2-43)
void hllc(const OCase &c, const Side &L, const Side &R, const double *YL, const double *YR, const double *S,
          double *F) {
  const double area = std::sqrt(((S[0]) * (S[0]) + (S[1]) * (S[1]) + (S[2]) * (S[2])));
  const double nx = S[0] / area, ny = S[1] / area, nz = S[2] / area;
  const double unL = ((L.u) * (S[0]) + (L.v) * (S[1]) + (L.w) * (S[2])) / area;
  const double unR = ((R.u) * (S[0]) + (R.v) * (S[1]) + (R.w) * (S[2])) / area;
  const double SL = unL - L.s.c, SR = unR + R.s.c;
  const double Sstar = (R.s.p - L.s.p + L.s.rho * unL * (SL - unL) - R.s.rho * unR * (SR - unR)) /
                       (L.s.rho * (SL - unL) - R.s.rho * (SR - unR));
  bool left, star;
  if (SL >= 0.0) left = true, star = false;
  else if (Sstar >= 0.0) left = true, star = true;
  else if (SR >= 0.0) left = false, star = true;
  else left = false, star = false;
  const Side &X = left ? L : R;
  const double *Y = left ? YL : YR;
  const double U = left ? unL : unR, SX = left ? SL : SR;
  const double et = X.s.e + 0.5 * ((X.u) * (X.u) + (X.v) * (X.v) + (X.w) * (X.w));
  const double mdot = U * X.s.rho * area;
  F[0] = mdot;
  F[1] = mdot * X.u + X.s.p * S[0];
  F[2] = mdot * X.v + X.s.p * S[1];
  F[3] = mdot * X.w + X.s.p * S[2];
  F[4] = mdot * et + U * X.s.p * area;
  for (int n = 0; n < c.ns - 1; n++) F[5 + n] = mdot * Y[n];
  if (star) {
    const double rhostar = X.s.rho * ((SX - U) / (SX - Sstar));
    const double drho = rhostar - X.s.rho, dU = rhostar * (Sstar - U);
    const double jump = SX * area;
    F[0] += jump * drho;
    F[1] += jump * (drho * X.u + dU * nx);
    F[2] += jump * (drho * X.v + dU * ny);
    F[3] += jump * (drho * X.w + dU * nz);
    F[4] += jump * (drho * et + dU * (Sstar + X.s.p / (X.s.rho * (SX - U))));
    for (int n = 0; n < c.ns - 1; n++) F[5 + n] += jump * drho * Y[n];
  }
}

// Rusanov with Davis's bound on the fastest wave (simulator/euler/kernels/flux/function/rusanov.mako:2-21)
void rusanov(const OCase &c, const Side &L, const Side &R, const double *YL, const double *YR, const double *S,
             double *F) {
  const double area = std::sqrt(((S[0]) * (S[0]) + (S[1]) * (S[1]) + (S[2]) * (S[2])));
  const double unL = ((L.u) * (S[0]) + (L.v) * (S[1]) + (L.w) * (S[2])) / area;
  const double unR = ((R.u) * (S[0]) + (R.v) * (S[1]) + (R.w) * (S[2])) / area;
  const double lam = std::fmax(std::fabs(unL) + L.s.c, std::fabs(unR) + R.s.c) * area;
  const double UL = unL * area, UR = unR * area;
  const double rL = L.s.rho, rR = R.s.rho, pL = L.s.p, pR = R.s.p;
  F[0] = 0.5 * (UR * rR + UL * rL - lam * (rR - rL));
  F[1] = 0.5 * (UR * rR * R.u + pR * S[0] + UL * rL * L.u + pL * S[0] - lam * (rR * R.u - rL * L.u));
  F[2] = 0.5 * (UR * rR * R.v + pR * S[1] + UL * rL * L.v + pL * S[1] - lam * (rR * R.v - rL * L.v));
  F[3] = 0.5 * (UR * rR * R.w + pR * S[2] + UL * rL * L.w + pL * S[2] - lam * (rR * R.w - rL * L.w));
  const double EL = rL * (L.s.e + 0.5 * ((L.u) * (L.u) + (L.v) * (L.v) + (L.w) * (L.w)));
  const double ER = rR * (R.s.e + 0.5 * ((R.u) * (R.u) + (R.v) * (R.v) + (R.w) * (R.w)));
  F[4] = 0.5 * (UR * (ER + pR) + UL * (EL + pL) - lam * (ER - EL));
  for (int n = 0; n < c.ns - 1; n++) {
    const double rhoYL = rL * YL[n], rhoYR = rR * YR[n];
    F[5 + n] = 0.5 * (rhoYR * UR + rhoYL * UL - lam * (rhoYR - rhoYL));
  }
}

// AUSM+-up of Liou (2006), cut-off Mach sqrt(0.1) (simulator/euler/kernels/flux/function/ausmup.mako:2-38)
void ausmup(const OCase &c, const Side &L, const Side &R, const double *YL, const double *YR, const double *S,
            double *F) {
  const double area = std::sqrt(((S[0]) * (S[0]) + (S[1]) * (S[1]) + (S[2]) * (S[2]))), invarea = 1.0 / area;
  const double UL = ((L.u) * (S[0]) + (L.v) * (S[1]) + (L.w) * (S[2])) * invarea;
  const double UR = ((R.u) * (S[0]) + (R.v) * (S[1]) + (R.w) * (S[2])) * invarea;
  const double a12 = 0.5 * (R.s.c + L.s.c), inva12 = 1.0 / a12;
  const double ML = UL * inva12, MR = UR * inva12;
  const double Mbarsq = 0.5 * (UL * UL + UR * UR) * inva12 * inva12;
  const double Mco = 0.31622776601683794, Kp = 0.25, Ku = 0.75, sigma = 1.0, beta = 1.0 / 8.0;
  const double Mo = std::sqrt(std::fmin(1.0, std::fmax(Mbarsq, Mco * Mco)));
  const double fa = Mo * (2.0 - Mo);
  const double M1p = 0.5 * (ML + std::fabs(ML)), M1m = 0.5 * (MR - std::fabs(MR));
  const double M2pL = 0.25 * (ML + 1.0) * (ML + 1.0), M2mL = -0.25 * (ML - 1.0) * (ML - 1.0);
  const double M2pR = 0.25 * (MR + 1.0) * (MR + 1.0), M2mR = -0.25 * (MR - 1.0) * (MR - 1.0);
  const double M4p = std::fabs(ML) >= 1.0 ? M1p : M2pL * (1.0 - 16.0 * beta * M2mL);
  const double M4m = std::fabs(MR) >= 1.0 ? M1m : M2mR * (1.0 + 16.0 * beta * M2pR);
  const double alpha = 3.0 / 16.0 * (-4.0 + 5.0 * fa * fa);
  const double p5p = std::fabs(ML) >= 1.0 ? (ML > 0.0 ? 1.0 : 0.0) : M2pL * ((2.0 - ML) - 16.0 * alpha * ML * M2mL);
  const double p5m = std::fabs(MR) >= 1.0 ? (MR < 0.0 ? 1.0 : 0.0) : M2mR * ((-2.0 - MR) + 16.0 * alpha * MR * M2pR);
  const double rho12 = 0.5 * (R.s.rho + L.s.rho);
  const double M12 = M4p + M4m - Kp * std::fmax(1.0 - sigma * Mbarsq, 0.0) * (R.s.p - L.s.p) * inva12 * inva12 / (fa * rho12);
  const double mdot = a12 * M12 * (M12 > 0.0 ? L.s.rho : R.s.rho) * area;
  const double p12 = p5p * L.s.p + p5m * R.s.p - Ku * p5p * p5m * (R.s.rho + L.s.rho) * fa * a12 * (UR - UL);
  const bool left = mdot > 0.0;
  const Side &U = left ? L : R;
  const double *Y = left ? YL : YR;
  F[0] = mdot;
  F[1] = mdot * U.u + p12 * S[0];
  F[2] = mdot * U.v + p12 * S[1];
  F[3] = mdot * U.w + p12 * S[2];
  F[4] = mdot * (U.s.e + 0.5 * ((U.u) * (U.u) + (U.v) * (U.v) + (U.w) * (U.w)) + U.s.p / U.s.rho);
  for (int n = 0; n < c.ns - 1; n++) F[5 + n] = mdot * Y[n];
}

// the double flux's Rusanov and AUSM+-up (simulator/eulerdf/kernels/flux/function/rusanov.mako:1-14,
// ausmup.mako:1-15): over the plain flux the energy row again in each cell's
// frozen plane, F[4] in the left's (recL) and F[ne] in the right's (recR),
// from each side's energy in that plane (eside,
// simulator/mixture/eos/realgasdf/kernels/eos.mako:73-83)
void riemann_df(const OCase &c, const Side &L, const Side &R, const double *YL, const double *YR, const double *S,
                const double *recL, const double *recR, double *F) {
  const int ns = c.ns, ne = 4 + ns;
  auto eside = [&](const Side &x, const double *Y, double *E) {
    for (int q = 0; q < 2; q++) {
      const double *pl = q == 0 ? recL : recR;
      double comp = 0.0;
      for (int n = 0; n < ns - 1; n++) comp += pl[S_ZETA + n] * Y[n];
      E[q] = pl[S_THETA] * x.s.p + x.s.rho * (pl[S_EPS] + comp + 0.5 * ((x.u) * (x.u) + (x.v) * (x.v) + (x.w) * (x.w))) +
             pl[S_KAPPA];
    }
  };
  if (c.primary == O_RUSANOV) {
    const double area = std::sqrt(((S[0]) * (S[0]) + (S[1]) * (S[1]) + (S[2]) * (S[2])));
    const double unL = ((L.u) * (S[0]) + (L.v) * (S[1]) + (L.w) * (S[2])) / area;
    const double unR = ((R.u) * (S[0]) + (R.v) * (S[1]) + (R.w) * (S[2])) / area;
    const double lam = std::fmax(std::fabs(unL) + L.s.c, std::fabs(unR) + R.s.c) * area;
    const double UL = unL * area, UR = unR * area;
    double EpL[2], EpR[2];
    eside(L, YL, EpL);
    eside(R, YR, EpR);
    for (int q = 0; q < 2; q++)
      F[q == 0 ? 4 : ne] = 0.5 * (UR * (EpR[q] + R.s.p) + UL * (EpL[q] + L.s.p) - lam * (EpR[q] - EpL[q]));
  } else {
    const double mdot = F[0];
    const bool left = mdot > 0.0;
    const Side &U = left ? L : R;
    const double rhoinvU = 1.0 / U.s.rho;
    double Ep[2];
    eside(U, left ? YL : YR, Ep);
    for (int q = 0; q < 2; q++) F[q == 0 ? 4 : ne] = mdot * (Ep[q] + U.s.p) * rhoinvU;
  }
}

// the advective flux of one face from its four cells (LL and RR read by MUSCL only):
// the reconstruction, then the flux function (simulator/euler/kernels/flux/single.mako:4-9);
// with the double flux's records of the two cells (recL, recR), its form
void advective(const OCase &c, const double *QLL, const double *QL, const double *QR, const double *QRR,
               const State &sLL, const State &sL, const State &sR, const State &sRR, const double *S, double *F,
               const double *recL = nullptr, const double *recR = nullptr) {
  double YL[16], YR[16];
  if (c.primary == O_KEPAEC) {
    kepaec(c, side(QL, sL), side(QR, sR), QL, QR, S, F);
    return;
  }
  Side L, R;
  if (c.recon == 1) {
    muscl(c, QLL, QL, QR, QRR, sLL, sL, sR, sRR, L, R, YL, YR);
  } else {
    L = side(QL, sL), R = side(QR, sR);
    for (int n = 0; n < c.ns - 1; n++) YL[n] = QL[5 + n] / QL[0], YR[n] = QR[5 + n] / QR[0];
  }
  if (c.primary == O_HLLC) hllc(c, L, R, YL, YR, S, F);
  else if (c.primary == O_RUSANOV) rusanov(c, L, R, YL, YR, S, F);
  else ausmup(c, L, R, YL, YR, S, F);
  if (recL) riemann_df(c, L, R, YL, YR, S, recL, recR, F);
}

// alpha damping (simulator/navstokes/kernels/flux/alpha-damping.mako:3-92)
void alphadamping(const OCase &c, const double *S, const double *xf, const double *xccL,
                  const double *xccR, const double *QL, const double *QR, const State &stateL,
                  const State &stateR, const double *trL, const double *trR, const double *hspL,
                  const double *hspR, const double *gL, const double *gR, double *F) {
  const int ns = c.ns;
  const double alpha = c.alpha, bulkvisc = 0.0;
  const double Sabs = std::sqrt(((S[0]) * (S[0]) + (S[1]) * (S[1]) + (S[2]) * (S[2]))), Sinv = 1.0 / Sabs;
  const double nx = S[0] * Sinv, ny = S[1] * Sinv, nz = S[2] * Sinv;
  const double mu = 0.5 * (trR[0] + trL[0]);
  const double kappa = 0.5 * (trR[1] + trL[1]);
  const double lambda = bulkvisc - 2.0 / 3.0 * mu;
  const double rhoinvL = stateL.rhoinv, rhoinvR = stateR.rhoinv;
  const double uL = QL[1] * rhoinvL, vL = QL[2] * rhoinvL, wL = QL[3] * rhoinvL;
  const double uR = QR[1] * rhoinvR, vR = QR[2] * rhoinvR, wR = QR[3] * rhoinvR;
  const double ex = xccR[0] - xccL[0], ey = xccR[1] - xccL[1], ez = xccR[2] - xccL[2];
  const double en0 = ex * nx, en1 = ey * ny, en2 = ez * nz;
  const double dampinv = alpha / std::sqrt(en0 * en0 + en1 * en1 + en2 * en2);
  const double dampx = dampinv * nx, dampy = dampinv * ny, dampz = dampinv * nz;
  const double xLx = xf[0] - xccL[0], xLy = xf[1] - xccL[1], xLz = xf[2] - xccL[2];
  const double xRx = xf[0] - xccR[0], xRy = xf[1] - xccR[1], xRz = xf[2] - xccR[2];
  auto facegrad = [&](int l, double phiL, double phiR, double &gx, double &gy, double &gz) {
    const double gLx = gL[3 * l + 0], gLy = gL[3 * l + 1], gLz = gL[3 * l + 2];
    const double gRx = gR[3 * l + 0], gRy = gR[3 * l + 1], gRz = gR[3 * l + 2];
    const double wl = phiL + gLx * xLx + gLy * xLy + gLz * xLz;
    const double wr = phiR + gRx * xRx + gRy * xRy + gRz * xRz;
    const double jump = wr - wl;
    gx = 0.5 * (gRx + gLx) + dampx * jump;
    gy = 0.5 * (gRy + gLy) + dampy * jump;
    gz = 0.5 * (gRz + gLz) + dampz * jump;
  };
  double dudx, dudy, dudz, dvdx, dvdy, dvdz, dwdx, dwdy, dwdz;
  facegrad(0, uL, uR, dudx, dudy, dudz);
  facegrad(1, vL, vR, dvdx, dvdy, dvdz);
  facegrad(2, wL, wR, dwdx, dwdy, dwdz);
  const double div = dudx + dvdy + dwdz;
  const double txx = -2.0 * mu * dudx - lambda * div;
  const double txy = -mu * (dvdx + dudy);
  const double txz = -mu * (dwdx + dudz);
  const double tyy = -2.0 * mu * dvdy - lambda * div;
  const double tyz = -mu * (dwdy + dvdz);
  const double tzz = -2.0 * mu * dwdz - lambda * div;
  F[1] += txx * S[0] + txy * S[1] + txz * S[2];
  F[2] += txy * S[0] + tyy * S[1] + tyz * S[2];
  F[3] += txz * S[0] + tyz * S[1] + tzz * S[2];
  double dTx, dTy, dTz;
  facegrad(3, stateL.T, stateR.T, dTx, dTy, dTz);
  const double heatflux = -kappa * (dTx * S[0] + dTy * S[1] + dTz * S[2]);
  const double uf = 0.5 * (uR + uL), vf = 0.5 * (vR + vL), wf = 0.5 * (wR + wL);
  double f4 = (uf * txx + vf * txy + wf * txz) * S[0] + (uf * txy + vf * tyy + wf * tyz) * S[1] +
              (uf * txz + vf * tyz + wf * tzz) * S[2] + heatflux;
  double YlastL = 1.0, YlastR = 1.0;
  for (int n = 0; n < ns - 1; n++) {
    YlastL -= QL[5 + n] * rhoinvL;
    YlastR -= QR[5 + n] * rhoinvR;
  }
  auto YL = [&](int n) { return n < ns - 1 ? QL[5 + n] * rhoinvL : YlastL; };
  auto YR = [&](int n) { return n < ns - 1 ? QR[5 + n] * rhoinvR : YlastR; };
  double Dk, Vc = 0.0, gradYns = 0.0, sumYh = 0.0, Yns = 1.0;
  const double rho = 0.5 * (QR[0] + QL[0]);
  for (int n = 0; n < ns - 1; n++) {
    Dk = 0.5 * (trR[2 + n] + trL[2 + n]);
    double dYx, dYy, dYz;
    facegrad(4 + n, YL(n), YR(n), dYx, dYy, dYz);
    const double gradYk = dYx * S[0] + dYy * S[1] + dYz * S[2];
    gradYns -= gradYk;
    Vc += Dk * gradYk;
    const double Jk = -rho * Dk * gradYk;
    const double hk = 0.5 * (hspR[n] + hspL[n]);
    const double Yk = 0.5 * (YR(n) + YL(n));
    Yns -= Yk;
    sumYh += Yk * hk;
    F[5 + n] += Jk;
    f4 += Jk * hk;
  }
  Dk = 0.5 * (trR[2 + ns - 1] + trL[2 + ns - 1]);
  Vc += Dk * gradYns;
  const double corr = rho * Vc;
  for (int n = 0; n < ns - 1; n++) F[5 + n] += 0.5 * (YR(n) + YL(n)) * corr;
  f4 += corr * sumYh;
  const double hns = 0.5 * (hspR[ns - 1] + hspL[ns - 1]);
  f4 += (-rho * Dk * gradYns + Yns * corr) * hns;
  F[4] += f4;
  // the double flux's second energy row takes the same diffusive energy flux
  // (simulator/navstokesdf/kernels/flux/alpha-damping.mako:1-9)
  if (c.df) F[4 + ns] += f4;
}

// the per-block scratch one right-hand side fills, as the reference's arrays
struct Scratch {
  std::vector<double> state, tr, hsp, grads, F[3];
};

// ---- boundaries: each kind's preadvflux on the halo cells behind its faces,
// the inflows' and outflows' postgrads, the walls' postflux
// (simulator/euler/kernels/bcs/*.mako, simulator/navstokes/kernels/bcs/*.mako,
// on the carried offsets of launch/policy.py:143-232: "interior" the first
// cell in whatever the layer, "mirror" layer l's image l deep, clamped to the
// block's depth, "mirror1" one deeper, "intface" the boundary face) ----
enum { B_SLIP_ADIA = 1, B_SLIP_ISOT, B_NOSLIP_ADIA, B_MOV_ADIA, B_NOSLIP_ISOT, B_MOV_ISOT, B_SUB_IN_FVT, B_SUP_IN_FA,
       B_SUB_IN_FTPTT, B_SUB_IN_FMT, B_SUB_OUT_FP, B_SUP_OUT_FN };

bool bc_wall(int kind) { return kind >= B_SLIP_ADIA && kind <= B_MOV_ISOT; }

// a boundary face's cells: the full index along its axis a of the cell d
// deep, of halo layer l and of the face; the in-plane axes a1 < a2
struct BFace {
  int a, a1, a2, g;
  bool low;
  int n[3];
  BFace(const OBlock &B, int nface) {
    a = (nface - 1) / 2;
    low = nface % 2 == 1;
    a1 = a == 0 ? 1 : 0;
    a2 = a == 2 ? 1 : 2;
    g = B.ng;
    n[0] = B.nx, n[1] = B.ny, n[2] = B.nz;
  }
  int deep(int d) const {
    d = std::min(d, n[a] - 1);
    return low ? g + d : g + n[a] - 1 - d;
  }
  int halo(int l) const { return low ? g - 1 - l : g + n[a] + l; }
  int face() const { return low ? g : g + n[a]; }
  long at(const Dims &d, int p, int q, int along) const {
    int c[3];
    c[a] = along, c[a1] = g + p, c[a2] = g + q;
    return d.at(c[0], c[1], c[2]);
  }
};

// fromprims into a cell's Q and record (simulator/euler/kernels/solution.mako:14-23)
void bc_fromprims(const OCase &c, double p, double T, const double *u, const double *Y, double *Q, double *rec) {
  double Z = 0.0;
  State th;
  if (c.realgas)
    th = rfrompT(c, p, T, [&](int n) { return Y[n]; }, Z);
  else
    th = frompT(c, p, T, Y);
  Q[0] = th.rho;
  Q[1] = th.rho * u[0];
  Q[2] = th.rho * u[1];
  Q[3] = th.rho * u[2];
  Q[4] = th.rho * (th.e + 0.5 * ((u[0]) * (u[0]) + (u[1]) * (u[1]) + (u[2]) * (u[2])));
  for (int n = 0; n < c.ns - 1; n++) Q[5 + n] = th.rho * Y[n];
  std::memcpy(rec, &th, sizeof(State));
  rec[S_Z] = Z;
}

// a face's unit normal scaled by sign (outward[0] for the outward one)
void unit_normal(const double *S, double sign, double *nrm) {
  const double Sinv = sign / std::sqrt((S[0]) * (S[0]) + (S[1]) * (S[1]) + (S[2]) * (S[2]));
  for (int d = 0; d < 3; d++) nrm[d] = S[d] * Sinv;
}

// the outflows' velocity (sub-out-fp.mako:17-30, sup-out-fn.mako:22-35)
void outflow_velocity(const double *Qi, double rhoinv, const double *Qm, const double *Qm1, const double *nrm,
                      double *u) {
  const double u0[3] = {Qi[1] * rhoinv, Qi[2] * rhoinv, Qi[3] * rhoinv};
  const double un = u0[0] * nrm[0] + u0[1] * nrm[1] + u0[2] * nrm[2];
  if (un > 0.0) {
    const double rhoinv1 = 1.0 / Qm1[0];
    for (int d = 0; d < 3; d++) u[d] = 2.0 * u0[d] - Qm1[1 + d] * rhoinv1;
  } else {
    const double rhoinvm = 1.0 / Qm[0];
    const double um[3] = {Qm[1] * rhoinvm, Qm[2] * rhoinvm, Qm[3] * rhoinvm};
    const double umn = 2.0 * (um[0] * nrm[0] + um[1] * nrm[1] + um[2] * nrm[2]);
    for (int d = 0; d < 3; d++) u[d] = um[d] - umn * nrm[d];
  }
}

// preadvflux of one boundary face: Q and the record of every halo cell behind it
void bc_halo(const OCase &c, OBlock &B, std::vector<double> &state, const OBc &bc) {
  const int ne = 4 + c.ns, ns = c.ns;
  const BFace w(B, bc.nface);
  const Dims d = cells(B), fd = face_dims(B, w.a);
  const double outward = w.low ? -1.0 : 1.0;
  for (int l = 0; l < B.ng; l++)
    for (int p = 0; p < w.n[w.a1]; p++)
      for (int q = 0; q < w.n[w.a2]; q++) {
        const double *v = bc.vals + ((long)p * w.n[w.a2] + q) * bc.nval;
        const long ci = w.at(d, p, q, w.deep(0)), cm = w.at(d, p, q, w.deep(l)), cm1 = w.at(d, p, q, w.deep(l + 1));
        const long ch = w.at(d, p, q, w.halo(l));
        const double *S = B.S[w.a] + w.at(fd, p, q, w.face()) * 3;
        const double *Qi = B.Q + ci * ne, *Qm = B.Q + cm * ne, *Qm1 = B.Q + cm1 * ne;
        const double *si = &state[ci * NSTATE], *sm = &state[cm * NSTATE], *sm1 = &state[cm1 * NSTATE];
        double *Qh = B.Q + ch * ne, *sh = &state[ch * NSTATE];
        double Y[16], u[3];
        switch (bc.kind) {
          case B_SLIP_ADIA: {  // slp-adia-wall.mako:4-22
            double nrm[3];
            unit_normal(S, 1.0, nrm);
            const double mn = 2.0 * (Qm[1] * nrm[0] + Qm[2] * nrm[1] + Qm[3] * nrm[2]);
            Qh[0] = Qm[0];
            for (int e = 0; e < 3; e++) Qh[1 + e] = Qm[1 + e] - mn * nrm[e];
            Qh[4] = Qm[4];
            for (int n = 0; n < ns - 1; n++) Qh[5 + n] = Qm[5 + n];
            std::memcpy(sh, sm, sizeof(double) * NSTATE);
            break;
          }
          case B_NOSLIP_ADIA:
          case B_MOV_ADIA: {  // navstokes/kernels/bcs/wall.mako:7-25, stuckhalo
            const bool mov = bc.kind == B_MOV_ADIA;
            const double rho = Qm[0], rhoinv = 1.0 / rho;
            double ke = 0.0, kehalo = 0.0;
            for (int e = 0; e < 3; e++) {
              const double ue = Qm[1 + e] * rhoinv, uh = 2.0 * (mov ? v[e] : 0.0) - ue;
              Qh[1 + e] = rho * uh;
              ke += ue * ue;
              kehalo += uh * uh;
            }
            Qh[0] = rho;
            Qh[4] = Qm[4] + 0.5 * rho * (kehalo - ke);
            for (int n = 0; n < ns - 1; n++) Qh[5 + n] = Qm[5 + n];
            std::memcpy(sh, sm, sizeof(double) * NSTATE);
            break;
          }
          case B_SLIP_ISOT: {  // slp-isot-wall.mako:5-20
            double nrm[3];
            unit_normal(S, 1.0, nrm);
            const double rhoinv = 1.0 / Qm[0];
            const double ui = Qm[1] * rhoinv, vi = Qm[2] * rhoinv, wi = Qm[3] * rhoinv;
            const double un = 2.0 * (ui * nrm[0] + vi * nrm[1] + wi * nrm[2]);
            u[0] = ui - un * nrm[0], u[1] = vi - un * nrm[1], u[2] = wi - un * nrm[2];
            for (int n = 0; n < ns - 1; n++) Y[n] = Qm[5 + n] * rhoinv;
            bc_fromprims(c, sm[0], v[0], u, Y, Qh, sh);
            break;
          }
          case B_NOSLIP_ISOT:
          case B_MOV_ISOT: {  // wall.mako:27-38, stuckhaloisot
            const bool mov = bc.kind == B_MOV_ISOT;
            const double rhoinv = 1.0 / Qm[0];
            for (int e = 0; e < 3; e++) u[e] = 2.0 * (mov ? v[e] : 0.0) - Qm[1 + e] * rhoinv;
            for (int n = 0; n < ns - 1; n++) Y[n] = Qm[5 + n] * rhoinv;
            bc_fromprims(c, sm[0], mov ? v[3] : v[0], u, Y, Qh, sh);
            break;
          }
          case B_SUB_IN_FVT: {  // sub-in-fvt.mako:4-14
            const double pp = 2.0 * si[0] - sm1[0];
            for (int e = 0; e < 3; e++) u[e] = v[e];
            for (int n = 0; n < ns - 1; n++) Y[n] = v[4 + n];
            bc_fromprims(c, pp, v[3], u, Y, Qh, sh);
            break;
          }
          case B_SUP_IN_FA: {  // sup-in-fa.mako:4-13
            for (int e = 0; e < 3; e++) u[e] = v[1 + e];
            for (int n = 0; n < ns - 1; n++) Y[n] = v[5 + n];
            bc_fromprims(c, v[0], v[4], u, Y, Qh, sh);
            break;
          }
          case B_SUB_IN_FMT: {  // sub-in-fmt.mako:4-30
            double nrm[3];
            unit_normal(S, -outward, nrm);
            const double pp = 2.0 * si[0] - sm1[0], T = v[1];
            for (int n = 0; n < ns - 1; n++) Y[n] = v[2 + n];
            double Z = 0.0;
            State th;
            if (c.realgas)
              th = rfrompT(c, pp, T, [&](int n) { return Y[n]; }, Z);
            else
              th = frompT(c, pp, T, Y);
            const double rhoinv = 1.0 / Qi[0];
            const double scale = 4.0 * v[0] / (Qi[0] + th.rho);
            for (int e = 0; e < 3; e++) u[e] = nrm[e] * scale - Qi[1 + e] * rhoinv;
            Qh[0] = th.rho;
            for (int e = 0; e < 3; e++) Qh[1 + e] = th.rho * u[e];
            Qh[4] = th.rho * (th.e + 0.5 * ((u[0]) * (u[0]) + (u[1]) * (u[1]) + (u[2]) * (u[2])));
            for (int n = 0; n < ns - 1; n++) Qh[5 + n] = th.rho * Y[n];
            std::memcpy(sh, &th, sizeof(State));
            sh[S_Z] = Z;
            break;
          }
          case B_SUB_IN_FTPTT: {  // sub-in-ftptt.mako:4-45
            double nrm[3];
            unit_normal(S, -outward, nrm);
            State sti;
            std::memcpy(&sti, si, sizeof(State));
            const double gamma = sti.gamma, cs = sti.c, gm1 = gamma - 1.0;
            const double rhoinv = 1.0 / Qi[0];
            const double u0[3] = {Qi[1] * rhoinv, Qi[2] * rhoinv, Qi[3] * rhoinv};
            for (int n = 0; n < ns - 1; n++) Y[n] = v[2 + n];
            const double Ttotal = v[1];
            const State total = frompT(c, sti.p, Ttotal, Y);
            const State cell = frompT(c, sti.p, sti.T, Y);
            const double Ht = cs * cs / gm1 + (total.e + total.p / total.rho) - (cell.e + cell.p / cell.rho);
            const double Un = u0[0] * nrm[0] + u0[1] * nrm[1] + u0[2] * nrm[2];
            const double Jm = -Un + 2.0 * cs / gm1;
            const double aq = 1.0 + 2.0 / gm1;
            const double bq = -2.0 * Jm;
            const double cq = gm1 * (0.5 * Jm * Jm - Ht);
            const double t1 = -bq / (2.0 * aq);
            const double t2 = std::sqrt(std::fmax(bq * bq - 4.0 * aq * cq, 0.0)) / (2.0 * aq);
            const double cb = std::fmax(t1 + t2, t1 - t2);
            const double Vb = 2.0 * cb / gm1 - Jm;
            const double Mb = Vb / cb;
            const double isentropic = 1.0 + 0.5 * gm1 * Mb * Mb;
            const double pp = v[0] * std::pow(isentropic, -gamma / gm1), T = Ttotal / isentropic;
            for (int e = 0; e < 3; e++) u[e] = Vb * nrm[e];
            bc_fromprims(c, pp, T, u, Y, Qh, sh);
            break;
          }
          case B_SUB_OUT_FP: {  // sub-out-fp.mako:4-41
            double nrm[3];
            unit_normal(S, outward, nrm);
            const double rhoinv = 1.0 / Qi[0];
            outflow_velocity(Qi, rhoinv, Qm, Qm1, nrm, u);
            for (int n = 0; n < ns - 1; n++) Y[n] = Qi[5 + n] * rhoinv;
            bc_fromprims(c, v[0], si[1], u, Y, Qh, sh);
            break;
          }
          case B_SUP_OUT_FN: {  // sup-out-fn.mako:4-48
            double nrm[3];
            unit_normal(S, outward, nrm);
            const double rhoinv = 1.0 / Qi[0], rhoinv1 = 1.0 / Qm1[0];
            const double least = 0.01, p0 = si[0], T0 = si[1];
            const double pp = std::fmin(std::fmax(least * p0, 2.0 * p0 - sm1[0]), p0);
            const double T = std::fmax(least * T0, 2.0 * T0 - sm1[1]);
            outflow_velocity(Qi, rhoinv, Qm, Qm1, nrm, u);
            for (int n = 0; n < ns - 1; n++)
              Y[n] = std::fmax(0.0, std::fmin(1.0, 2.0 * Qi[5 + n] * rhoinv - Qm1[5 + n] * rhoinv1));
            bc_fromprims(c, pp, T, u, Y, Qh, sh);
            break;
          }
          default: break;
        }
        if (B.Tg) B.Tg[ch] = sh[1];
      }
}

// postgrads of an inflow or outflow: the halo's gradients its image's
// (navstokes/kernels/bcs/gradients.mako:2-6)
void bc_grads(const OBlock &B, double *grads, int ngrad, const OBc &bc) {
  const BFace w(B, bc.nface);
  const Dims d = cells(B);
  for (int l = 0; l < B.ng; l++)
    for (int p = 0; p < w.n[w.a1]; p++)
      for (int q = 0; q < w.n[w.a2]; q++) {
        const long cm = w.at(d, p, q, w.deep(l)), ch = w.at(d, p, q, w.halo(l));
        std::memcpy(&grads[ch * ngrad * 3], &grads[cm * ngrad * 3], sizeof(double) * ngrad * 3);
      }
}

// postflux of a wall: the face flux from the first cell in, over the flux
// function's (euler/kernels/bcs/wall.mako:2-16; with viscosity
// navstokes/kernels/bcs/wall.mako:40-99)
void bc_wallflux(const OCase &c, const OBlock &B, const std::vector<double> &state, const std::vector<double> &tr,
                 std::vector<double> &F, int nf, const OBc &bc) {
  const int ne = 4 + c.ns, ns = c.ns;
  const bool visc = c.simulator == O_NAVSTOKES;
  const BFace w(B, bc.nface);
  const Dims d = cells(B), fd = face_dims(B, w.a);
  const double outward = w.low ? -1.0 : 1.0;
  const bool mov = bc.kind == B_MOV_ADIA || bc.kind == B_MOV_ISOT;
  const bool isot = bc.kind == B_SLIP_ISOT || bc.kind == B_NOSLIP_ISOT || bc.kind == B_MOV_ISOT;
  const double stuck = (bc.kind == B_SLIP_ADIA || bc.kind == B_SLIP_ISOT) ? 0.0 : 1.0;
  for (int p = 0; p < w.n[w.a1]; p++)
    for (int q = 0; q < w.n[w.a2]; q++) {
      const double *v = bc.vals + ((long)p * w.n[w.a2] + q) * bc.nval;
      const long fi = w.at(fd, p, q, w.face()), ci = w.at(d, p, q, w.deep(0));
      const double *S = B.S[w.a] + fi * 3, *xf = B.xf[w.a] + fi * 3, *xcc = B.xcc + ci * 3;
      const double *Q = B.Q + ci * ne;
      State st;
      std::memcpy(&st, &state[ci * NSTATE], sizeof(State));
      double *Fo = &F[fi * nf];
      // wallpressure and wallflux
      const double area = std::sqrt((S[0]) * (S[0]) + (S[1]) * (S[1]) + (S[2]) * (S[2]));
      const double un = outward * ((Q[1]) * (S[0]) + (Q[2]) * (S[1]) + (Q[3]) * (S[2])) / (Q[0] * area);
      const double pw = std::fmax(st.p + Q[0] * st.c * un, 0.0);
      Fo[0] = 0.0;
      for (int e = 0; e < 3; e++) Fo[1 + e] = pw * S[e];
      for (int l = 4; l < nf; l++) Fo[l] = 0.0;
      if (!visc) continue;
      const double wall[3] = {mov ? v[0] : 0.0, mov ? v[1] : 0.0, mov ? v[2] : 0.0};
      double mu, kappa, dT;
      if (isot) {
        // wallcoeffs at the wall's temperature and the first cell's pressure and composition
        const double Tw = bc.kind == B_MOV_ISOT ? v[3] : v[0];
        const double rhoinv = 1.0 / Q[0];
        double Y[16], trw[2 + 16], hw[16];
        for (int n = 0; n < ns - 1; n++) Y[n] = Q[5 + n] * rhoinv;
        const State at = frompT(c, st.p, Tw, Y);
        transport(c, Q, at, trw, hw);
        mu = trw[0], kappa = trw[1], dT = Tw - st.T;
      } else {
        mu = tr[ci * (2 + ns)], kappa = tr[ci * (2 + ns) + 1], dT = 0.0;
      }
      const double Sabs = area, Sinv = 1.0 / Sabs;
      const double n[3] = {S[0] * Sinv, S[1] * Sinv, S[2] * Sinv};
      const double dn = std::fabs(((xcc[0] - xf[0])) * (n[0]) + ((xcc[1] - xf[1])) * (n[1]) + ((xcc[2] - xf[2])) * (n[2]));
      const double rhoinv = 1.0 / Q[0];
      double dun[3];
      for (int e = 0; e < 3; e++) dun[e] = outward * (wall[e] - Q[1 + e] * rhoinv) / dn;
      const double div = (dun[0]) * (n[0]) + (dun[1]) * (n[1]) + (dun[2]) * (n[2]);
      for (int e = 0; e < 3; e++) dun[e] = div * n[e] + stuck * (dun[e] - div * n[e]);
      double work = 0.0;
      for (int e = 0; e < 3; e++) {
        const double tS = -mu * Sabs * (dun[e] + div * n[e] / 3.0);
        Fo[1 + e] += tS;
        work += wall[e] * tS;
      }
      Fo[4] += work - kappa * outward * (dT) / dn * Sabs;
      // the double flux's second energy row: nothing is advected through a
      // wall, so it is the first's (simulator/navstokesdf/kernels/bcs/*-wall.mako)
      if (nf > ne) Fo[ne] = Fo[4];
    }
}

// a three-vector at stride st turned by R (place.mako:4-9)
void rotate3(double *x, int st, const double *R) {
  const double a = x[0], b = x[st], c = x[2 * st];
  x[0] = R[0] * a + R[1] * b + R[2] * c;
  x[st] = R[3] * a + R[4] * b + R[5] * c;
  x[2 * st] = R[6] * a + R[7] * b + R[8] * c;
}

// the turn a rotational periodic gives what lands in its halo: the vector at
// component vec (Q's momentum at 1), or with vec -2 the gradients' tensor,
// each row's directions and then the velocity rows down every direction
// (simulator place.mako:11-36)
void rotate_cell(const OCase &c, const OHaloEntry &h, double *dp, int comps, int vec) {
  if (!h.rot || !c.rots || vec == -1) return;
  const double *R = c.rots + 9 * (h.rot - 1);
  if (vec >= 0) {
    rotate3(dp + vec, 1, R);
    return;
  }
  for (int r = 0; r < comps / 3; r++) rotate3(dp + 3 * r, 1, R);
  for (int m = 0; m < 3; m++) rotate3(dp + m, 3, R);
}

void halo_fill(const OCase &c, std::vector<OBlock> &blks, const OHaloEntry *map, long nmap, int maxlayer, int comps,
               int vec, double *(*arr)(OBlock &, std::vector<Scratch> &, int), std::vector<Scratch> &scr) {
  for (long m = 0; m < nmap; m++) {
    const OHaloEntry &h = map[m];
    if (h.layer >= maxlayer) continue;
    OBlock &d = blks[h.dblk];
    OBlock &s = blks[h.sblk];
    double *dp = arr(d, scr, h.dblk) + cells(d).at(h.di, h.dj, h.dk) * comps;
    const double *sp = arr(s, scr, h.sblk) + cells(s).at(h.si, h.sj, h.sk) * comps;
    std::memcpy(dp, sp, sizeof(double) * comps);
    rotate_cell(c, h, dp, comps, vec);
  }
}

}  // namespace

extern "C" {

// The right-hand side of every block: dQ = the flux divergence of Q.
// prerhs: Q's halo exchanged, fromQ everywhere it is read, transport on the
// interior and first halo layer; rhs: gradients on the interior and their
// one-plane exchange, advective then diffusive face fluxes on the interior
// faces, applyflux (simulator/advec/kernels/applyflux.mako:2-11).
// faces, when not null, receives each block's face fluxes: faces[3 b + a] the
// array of axis a, [X'][Y'][Z'][ne] with one plane more along a.
int oracle_rhs(const OCase *cp, OBlock *blocks, int nblocks, const OHaloEntry *map, long nmap,
               double **dQ, double **faces) {
  const OCase &c = *cp;
  const int ns = c.ns, ne = 4 + ns, ngrad = ne - 1;
  const bool visc = c.simulator == O_NAVSTOKES;
  std::vector<OBlock> blks(blocks, blocks + nblocks);
  std::vector<Scratch> scr(nblocks);
  // Q's halo: every layer (simulator/advec/simulator.py:57-63)
  halo_fill(c, blks, map, nmap, 1 << 30, ne, 1, [](OBlock &b, std::vector<Scratch> &, int) { return b.Q; }, scr);
  for (int b = 0; b < nblocks; b++) {
    OBlock &B = blks[b];
    const Dims d = cells(B);
    const long N = (long)d.X * d.Y * d.Z;
    Scratch &s = scr[b];
    s.state.assign(N * NSTATE, 0.0);
    s.tr.assign(N * (2 + ns), 0.0);
    s.hsp.assign(N * ns, 0.0);
    s.grads.assign(N * ngrad * 3, 0.0);
    // the state wherever Q is set: interior and the face halos (edges and
    // corners of the halo hold no density and are never read)
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < d.X; i++)
      for (int j = 0; j < d.Y; j++)
        for (int k = 0; k < d.Z; k++) {
          const int out = (i < B.ng || i >= d.X - B.ng) + (j < B.ng || j >= d.Y - B.ng) +
                          (k < B.ng || k >= d.Z - B.ng);
          if (out > 1) continue;
          const long at = d.at(i, j, k);
          State st;
          if (c.realgas) {
            // the real gas's record: the state, Z and, with the double flux,
            // the cell's frozen plane kept across stages
            double *rec = &s.state[at * NSTATE];
            if (c.df) std::memcpy(rec, B.pst + at * NSTATE, sizeof(double) * NSTATE);
            rstate(c, B.Q + at * ne, rec, B.Tg ? B.Tg[at] : 0.0, c.df != 0);
            std::memcpy(&st, rec, sizeof(State));
            if (c.df) std::memcpy(B.pst + at * NSTATE, rec, sizeof(double) * NSTATE);
          } else {
            st = fromQ(c, B.Q + at * ne, B.Tg ? B.Tg[at] : 0.0);
            std::memcpy(&s.state[at * NSTATE], &st, sizeof(State));
          }
          if (B.Tg) B.Tg[at] = st.T;
        }
  }
  // the boundaries' halo cells, after the state they read and before the
  // transport reads theirs (simulator/advec/simulator.py:57-75)
  for (int m = 0; m < c.nbc; m++) bc_halo(c, blks[c.bc[m].blk], scr[c.bc[m].blk].state, c.bc[m]);
  for (int b = 0; b < nblocks; b++) {
    OBlock &B = blks[b];
    const Dims d = cells(B);
    Scratch &s = scr[b];
    if (visc) {
      // the shallow range: interior plus one halo layer
#pragma omp parallel for collapse(2) schedule(static)
      for (int i = 0; i < d.X; i++)
        for (int j = 0; j < d.Y; j++)
          for (int k = 0; k < d.Z; k++) {
            const int out = (i < B.ng || i >= d.X - B.ng) + (j < B.ng || j >= d.Y - B.ng) +
                            (k < B.ng || k >= d.Z - B.ng);
            const int deep = (i < B.ng - 1 || i > d.X - B.ng) + (j < B.ng - 1 || j > d.Y - B.ng) +
                             (k < B.ng - 1 || k > d.Z - B.ng);
            if (out > 1 || deep) continue;
            const long at = d.at(i, j, k);
            State st;
            std::memcpy(&st, &s.state[at * NSTATE], sizeof(State));
            transport(c, B.Q + at * ne, st, &s.tr[at * (2 + ns)], &s.hsp[at * ns], s.state[at * NSTATE + S_Z]);
          }
    }
    if (visc) {
      // dqdxyz (simulator/navstokes/kernels/dqdxyz.mako:16-41) on the interior
#pragma omp parallel for collapse(2) schedule(static)
      for (int i = B.ng; i < d.X - B.ng; i++)
        for (int j = B.ng; j < d.Y - B.ng; j++)
          for (int k = B.ng; k < d.Z - B.ng; k++) {
            const long at = d.at(i, j, k);
            const double *QpI = B.Q + d.at(i + 1, j, k) * ne, *QmI = B.Q + d.at(i - 1, j, k) * ne;
            const double *QpJ = B.Q + d.at(i, j + 1, k) * ne, *QmJ = B.Q + d.at(i, j - 1, k) * ne;
            const double *QpK = B.Q + d.at(i, j, k + 1) * ne, *QmK = B.Q + d.at(i, j, k - 1) * ne;
            const double TpI = s.state[d.at(i + 1, j, k) * NSTATE + 1], TmI = s.state[d.at(i - 1, j, k) * NSTATE + 1];
            const double TpJ = s.state[d.at(i, j + 1, k) * NSTATE + 1], TmJ = s.state[d.at(i, j - 1, k) * NSTATE + 1];
            const double TpK = s.state[d.at(i, j, k + 1) * NSTATE + 1], TmK = s.state[d.at(i, j, k - 1) * NSTATE + 1];
            const double *J = B.Jinv + at * 9;
            double *g = &s.grads[at * ngrad * 3];
            const double rIp = QpI[0], rIm = QmI[0], invI = 1.0 / (rIp * rIm);
            const double rJp = QpJ[0], rJm = QmJ[0], invJ = 1.0 / (rJp * rJm);
            const double rKp = QpK[0], rKm = QmK[0], invK = 1.0 / (rKp * rKm);
            auto phys = [&](int l, const double *dd) {
              for (int e = 0; e < 3; e++) g[3 * l + e] = dd[0] * J[0 * 3 + e] + dd[1] * J[1 * 3 + e] + dd[2] * J[2 * 3 + e];
            };
            for (int l = 0; l < ngrad; l++) {
              if (l == 3) {
                const double dd[3] = {0.5 * (TpI - TmI), 0.5 * (TpJ - TmJ), 0.5 * (TpK - TmK)};
                phys(l, dd);
                continue;
              }
              const int m = l + 1;
              const double dd[3] = {0.5 * (QpI[m] * rIm - QmI[m] * rIp) * invI,
                                    0.5 * (QpJ[m] * rJm - QmJ[m] * rJp) * invJ,
                                    0.5 * (QpK[m] * rKm - QmK[m] * rKp) * invK};
              phys(l, dd);
            }
          }
    }
  }
  if (visc) {
    // grads: one halo plane (simulator/advecdiff/simulator.py:11-14, 116-117)
    halo_fill(c, blks, map, nmap, 1, ngrad * 3, -2,
              [](OBlock &, std::vector<Scratch> &s, int b) { return s[b].grads.data(); }, scr);
    // the inflows' and outflows' halo gradients (simulator/advecdiff/simulator.py:113-114)
    for (int m = 0; m < c.nbc; m++)
      if (!bc_wall(c.bc[m].kind)) bc_grads(blks[c.bc[m].blk], scr[c.bc[m].blk].grads.data(), ngrad, c.bc[m]);
  }
  const int nf = ne + (c.df ? 1 : 0);
  for (int b = 0; b < nblocks; b++) {
    OBlock &B = blks[b];
    const Dims d = cells(B);
    Scratch &s = scr[b];
    const int g = B.ng;
    // the double flux writes its energy row twice: one row more per face
    for (int a = 0; a < 3; a++) {
      const Dims f = face_dims(B, a);
      s.F[a].assign((long)f.X * f.Y * f.Z * nf, 0.0);
      const int hi[3] = {B.nx + (a == 0), B.ny + (a == 1), B.nz + (a == 2)};
      // the interior faces of axis a: a face is indexed like the cell to its right
      // (peregrine/launch/policy.py:78-86)
#pragma omp parallel for collapse(2) schedule(static)
      for (int i = g; i < g + hi[0]; i++)
        for (int j = g; j < g + hi[1]; j++)
          for (int k = g; k < g + hi[2]; k++) {
            const long at = f.at(i, j, k);
            const long R = d.at(i, j, k);
            const long L = d.at(i - (a == 0), j - (a == 1), k - (a == 2));
            const long LL = d.at(i - 2 * (a == 0), j - 2 * (a == 1), k - 2 * (a == 2));
            const long RR = d.at(i + (a == 0), j + (a == 1), k + (a == 2));
            const double *QL = B.Q + L * ne, *QR = B.Q + R * ne;
            const State &sL = *reinterpret_cast<const State *>(&s.state[L * NSTATE]);
            const State &sR = *reinterpret_cast<const State *>(&s.state[R * NSTATE]);
            const State &sLL = *reinterpret_cast<const State *>(&s.state[LL * NSTATE]);
            const State &sRR = *reinterpret_cast<const State *>(&s.state[RR * NSTATE]);
            double *F = &s.F[a][at * nf];
            const double *S = B.S[a] + at * 3;
            if (c.df && c.primary == O_KEPAEC)
              kepaec_df(c, QL, QR, &s.state[L * NSTATE], &s.state[R * NSTATE], S, F);
            else if (c.df)
              advective(c, B.Q + LL * ne, QL, QR, B.Q + RR * ne, sLL, sL, sR, sRR, S, F, &s.state[L * NSTATE],
                        &s.state[R * NSTATE]);
            else if (!c.skip_adv)
              advective(c, B.Q + LL * ne, QL, QR, B.Q + RR * ne, sLL, sL, sR, sRR, S, F);
            if (visc)
              alphadamping(c, S, B.xf[a] + at * 3, B.xcc + L * 3, B.xcc + R * 3, QL, QR, sL, sR,
                           &s.tr[L * (2 + ns)], &s.tr[R * (2 + ns)], &s.hsp[L * ns], &s.hsp[R * ns],
                           &s.grads[L * ngrad * 3], &s.grads[R * ngrad * 3], F);
          }
    }
  }
  // the walls write the flux through their faces over the flux function's
  // (simulator/advec/simulator.py:80-84)
  for (int m = 0; m < c.nbc; m++) {
    const OBc &bc = c.bc[m];
    if (!bc_wall(bc.kind)) continue;
    const int a = (bc.nface - 1) / 2;
    bc_wallflux(c, blks[bc.blk], scr[bc.blk].state, scr[bc.blk].tr, scr[bc.blk].F[a], nf, bc);
  }
  for (int b = 0; b < nblocks; b++) {
    OBlock &B = blks[b];
    const Dims d = cells(B);
    Scratch &s = scr[b];
    const int g = B.ng;
    if (faces)
      for (int a = 0; a < 3; a++) std::memcpy(faces[3 * b + a], s.F[a].data(), sizeof(double) * s.F[a].size());
    const Dims fi = face_dims(B, 0), fj = face_dims(B, 1), fk = face_dims(B, 2);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = g; i < g + B.nx; i++)
      for (int j = g; j < g + B.ny; j++)
        for (int k = g; k < g + B.nz; k++) {
          const double *iFl = &s.F[0][fi.at(i, j, k) * nf], *iFh = &s.F[0][fi.at(i + 1, j, k) * nf];
          const double *jFl = &s.F[1][fj.at(i, j, k) * nf], *jFh = &s.F[1][fj.at(i, j + 1, k) * nf];
          const double *kFl = &s.F[2][fk.at(i, j, k) * nf], *kFh = &s.F[2][fk.at(i, j, k + 1) * nf];
          const long at = d.at(i, j, k);
          const double detJinv = B.detJinv[at];
          if (c.df) {
            // the cell's own energy row: F[ne] on its low faces, where it is the
            // right cell, F[4] on its high faces (simulator/eulerdf/kernels/applyflux.mako:2-14)
            for (int l = 0; l < ne; l++) {
              if (l == 4) continue;
              dQ[b][at * ne + l] = (iFl[l] + jFl[l] + kFl[l] - iFh[l] - jFh[l] - kFh[l]) * detJinv;
            }
            dQ[b][at * ne + 4] = (iFl[ne] + jFl[ne] + kFl[ne] - iFh[4] - jFh[4] - kFh[4]) * detJinv;
          } else if (c.mech) {
            // coupled chemistry begins dQ with the carried species' production
            // rates, the fluxes add to it (simulator/chemint/kernels/source.mako:3-10,
            // cell.mako:14-19, applyflux.mako with append)
            double omega[16], src[32];
            if (c.substepped) {
              const int taken = substepped(c, B.Q + at * ne, s.state[at * NSTATE + 1], omega);
              if (B.subs) B.subs[at] = taken;
            } else {
              cellrates(c, B.Q + at * ne, s.state[at * NSTATE + 1], omega);
            }
            for (int l = 0; l < 5; l++) src[l] = 0.0;
            for (int n = 0; n < ns - 1; n++) src[5 + n] = omega[n];
            for (int l = 0; l < ne; l++)
              dQ[b][at * ne + l] = src[l] + (iFl[l] + jFl[l] + kFl[l] - iFh[l] - jFh[l] - kFh[l]) * detJinv;
          } else {
            for (int l = 0; l < ne; l++)
              dQ[b][at * ne + l] = (iFl[l] + jFl[l] + kFl[l] - iFh[l] - jFh[l] - kFh[l]) * detJinv;
          }
        }
  }
  return 0;
}

// the transport state (mu, kappa, D[ns]) of n cells: Q rows and their
// states (EosState rows, 8 wide); tr [n][2 + ns]
int oracle_transport(const OCase *cp, long n, const double *Q, const double *st, double *tr) {
  const OCase &c = *cp;
  const int ne = 4 + c.ns;
  std::vector<double> h(c.ns);
  for (long q = 0; q < n; q++) {
    State s;
    std::memcpy(&s, st + q * 8, sizeof(State));
    transport(c, Q + q * ne, s, tr + q * (2 + c.ns), h.data());
  }
  return 0;
}

// cflmax over every block's interior (simulator/euler/kernels/cflmax.mako:2-33
// with the cell lengths of multiblock/block/grid.py:164-176): the largest
// acoustic, convective and combined CFL number per unit step, out[3]; the
// state from Q as the stage's fromQ makes it (the cell's Tg as the guess)
int oracle_cflmax(const OCase *cp, const OBlock *blocks, int nblocks, double *out) {
  const OCase &c = *cp;
  const int ne = 4 + c.ns;
  double m[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < nblocks; b++) {
    const OBlock &B = blocks[b];
    const Dims d = cells(B);
    const int n[3] = {B.nx, B.ny, B.nz};
    const int g = B.ng;
    for (int i = g; i < g + B.nx; i++)
      for (int j = g; j < g + B.ny; j++)
        for (int k = g; k < g + B.nz; k++) {
          const long at = d.at(i, j, k);
          const double *Q = B.Q + at * ne;
          State st;
          if (c.realgas) {
            double rec[NSTATE] = {};
            if (c.df) std::memcpy(rec, B.pst + at * NSTATE, sizeof(double) * NSTATE);
            rstate(c, Q, rec, B.Tg ? B.Tg[at] : 0.0, c.df != 0);
            std::memcpy(&st, rec, sizeof(State));
          } else {
            st = fromQ(c, Q, B.Tg ? B.Tg[at] : 0.0);
          }
          const double rhoinv = 1.0 / Q[0];
          const double u = Q[1] * rhoinv, v = Q[2] * rhoinv, w = Q[3] * rhoinv;
          double dl[3], un[3];
          for (int a = 0; a < 3; a++) {
            const Dims f = face_dims(B, a);
            const long lo = f.at(i, j, k), hi = f.at(i + (a == 0), j + (a == 1), k + (a == 2));
            const double *L = B.S[a] + lo * 3, *H = B.S[a] + hi * 3;
            const double *xl = B.xf[a] + lo * 3, *xh = B.xf[a] + hi * 3;
            const double s0 = xh[0] - xl[0], s1 = xh[1] - xl[1], s2 = xh[2] - xl[2];
            // an axis one cell thick is not marched in: infinitely long
            dl[a] = n[a] == 1 ? INFINITY : std::sqrt(s0 * s0 + s1 * s1 + s2 * s2);
            const double S0inv = 1.0 / std::sqrt((L[0]) * (L[0]) + (L[1]) * (L[1]) + (L[2]) * (L[2]));
            const double S1inv = 1.0 / std::sqrt((H[0]) * (H[0]) + (H[1]) * (H[1]) + (H[2]) * (H[2]));
            const double nx = 0.5 * (L[0] * S0inv + H[0] * S1inv);
            const double ny = 0.5 * (L[1] * S0inv + H[1] * S1inv);
            const double nz = 0.5 * (L[2] * S0inv + H[2] * S1inv);
            un[a] = std::fabs(nx * u + ny * v + nz * w);
          }
          const double acoustic = st.c * std::sqrt(1.0 / (dl[0] * dl[0]) + 1.0 / (dl[1] * dl[1]) + 1.0 / (dl[2] * dl[2]));
          const double convective = un[0] / dl[0] + un[1] / dl[1] + un[2] / dl[2];
          m[0] = std::fmax(m[0], acoustic);
          m[1] = std::fmax(m[1], convective);
          m[2] = std::fmax(m[2], acoustic + convective);
        }
  }
  for (int q = 0; q < 3; q++) out[q] = m[q];
  return 0;
}

// The boundaries' gradient hook alone on given gradient arrays, grads[b]
// [..][ngrad][3] over block b's full extents (the reference's postgrads)
int oracle_bc_grads(const OCase *cp, const OBlock *blocks, double **grads) {
  const OCase &c = *cp;
  for (int m = 0; m < c.nbc; m++)
    if (!bc_wall(c.bc[m].kind)) bc_grads(blocks[c.bc[m].blk], grads[c.bc[m].blk], 3 + c.ns, c.bc[m]);
  return 0;
}

// The double flux's step start on register Q: each interior cell's state
// (the real gas's fromrhoE when first, else off its frozen plane), its plane
// frozen anew with the energy reset to the eos's, then Q, the kept records
// and the starting guesses copied into every halo layer, so a halo's plane is
// its image's (simulator/eulerdf/simulator.py:58-66, freeze.mako:3-32)
int oracle_prestep(const OCase *cp, OBlock *blocks, int nblocks, const OHaloEntry *map, long nmap, int first) {
  const OCase &c = *cp;
  const int ne = 4 + c.ns;
  for (int b = 0; b < nblocks; b++) {
    OBlock &B = blocks[b];
    const Dims d = cells(B);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = B.ng; i < d.X - B.ng; i++)
      for (int j = B.ng; j < d.Y - B.ng; j++)
        for (int k = B.ng; k < d.Z - B.ng; k++) {
          const long at = d.at(i, j, k);
          double *rec = B.pst + at * NSTATE;
          rstate(c, B.Q + at * ne, rec, B.Tg[at], !first);
          B.Tg[at] = rec[1];
          freeze(c, B.Q + at * ne, rec);
        }
  }
  for (long m = 0; m < nmap; m++) {
    const OHaloEntry &h = map[m];
    OBlock &D = blocks[h.dblk];
    OBlock &S = blocks[h.sblk];
    const long dt = cells(D).at(h.di, h.dj, h.dk), st = cells(S).at(h.si, h.sj, h.sk);
    std::memcpy(D.Q + dt * ne, S.Q + st * ne, sizeof(double) * ne);
    rotate_cell(c, h, D.Q + dt * ne, ne, 1);
    std::memcpy(D.pst + dt * NSTATE, S.pst + st * NSTATE, sizeof(double) * NSTATE);
    D.Tg[dt] = S.Tg[st];
  }
  // the boundaries' halo cells from the state just formed, then frozen like
  // every other cell (simulator/eulerdf/simulator.py:58-66 freezes "all")
  for (int m = 0; m < c.nbc; m++) {
    const OBc &bc = c.bc[m];
    OBlock &B = blocks[bc.blk];
    const Dims d = cells(B);
    const long N = (long)d.X * d.Y * d.Z;
    std::vector<double> state(B.pst, B.pst + N * NSTATE);
    bc_halo(c, B, state, bc);
    std::memcpy(B.pst, state.data(), sizeof(double) * N * NSTATE);
    const BFace w(B, bc.nface);
    for (int l = 0; l < B.ng; l++)
      for (int p = 0; p < w.n[w.a1]; p++)
        for (int q = 0; q < w.n[w.a2]; q++) {
          const long ch = w.at(d, p, q, w.halo(l));
          freeze(c, B.Q + ch * ne, B.pst + ch * NSTATE);
        }
  }
  return 0;
}

// the real gas's state at n (p, T, Y of the carried species) points by
// frompT, records [n][NSTATE] (Z at S_Z)
int oracle_realgas_frompT(const OCase *cp, long n, const double *p, const double *T, const double *Y, double *rec) {
  const int ns = cp->ns;
  for (long q = 0; q < n; q++) {
    double Z;
    const State s = rfrompT(*cp, p[q], T[q], [&](int k) { return Y[q * (ns - 1) + k]; }, Z);
    std::memcpy(rec + q * NSTATE, &s, sizeof(State));
    rec[q * NSTATE + S_Z] = Z;
  }
  return 0;
}

// the real gas's state at n (Q, T guess) by fromrhoE, records [n][NSTATE]
int oracle_realgas_fromQ(const OCase *cp, long n, const double *Q, const double *Tg, double *rec) {
  const int ne = 4 + cp->ns;
  for (long q = 0; q < n; q++) rstate(*cp, Q + q * ne, rec + q * NSTATE, Tg[q], false);
  return 0;
}

// freeze at n cells (Q rows, records from the eos): Q's energy and the planes in place
int oracle_freeze(const OCase *cp, long n, double *Q, double *rec) {
  const int ne = 4 + cp->ns;
  for (long q = 0; q < n; q++) freeze(*cp, Q + q * ne, rec + q * NSTATE);
  return 0;
}

// kepaec on n independent faces: each side's state from its Q by fromQ,
// rows [n][ne] (the flux-function check against the reference's numpy oracle)
int oracle_kepaec_faces(const OCase *cp, long n, const double *QL, const double *QR, const double *S, double *F) {
  const int ne = 4 + cp->ns;
  for (long f = 0; f < n; f++) {
    const double *ql = QL + f * ne, *qr = QR + f * ne;
    const State sl = fromQ(*cp, ql), sr = fromQ(*cp, qr);
    kepaec(*cp, side(ql, sl), side(qr, sr), ql, qr, S + 3 * f, F + f * ne);
  }
  return 0;
}

// the advective flux on n independent faces from the four cells around each,
// Q rows [4][n][ne] in the order LL, L, R, RR (the reconstruction and flux
// function check against the reference's numpy oracle)
int oracle_advective_faces(const OCase *cp, long n, const double *Q4, const double *S, double *F) {
  const int ne = 4 + cp->ns;
  for (long f = 0; f < n; f++) {
    const double *q[4];
    State st[4];
    for (int o = 0; o < 4; o++) q[o] = Q4 + ((long)o * n + f) * ne, st[o] = fromQ(*cp, q[o]);
    advective(*cp, q[0], q[1], q[2], q[3], st[0], st[1], st[2], st[3], S + 3 * f, F + f * ne);
  }
  return 0;
}

// fromprims over every cell a block has (interior and halos); Tg, when not
// null, receives each cell's stored T (the next fromQ's starting guess)
int oracle_fromprims(const OCase *cp, const double *q, double *Q, long ncells, double *Tg) {
  const int ne = 4 + cp->ns;
#pragma omp parallel for schedule(static)
  for (long n = 0; n < ncells; n++) {
    const double T = fromprims(*cp, q + n * ne, Q + n * ne);
    if (Tg) Tg[n] = T;
  }
  return 0;
}

// the production rates of n independent states (rho, Y[ns] every species, T)
// as the kernels form them: the rate state straight from Y, without the
// clipping cellrates applies (the reference's numpy twin's view,
// tests/mixture/rates.py:169-185)
int oracle_production(const OCase *cp, long n, const double *rho, const double *Y, const double *T,
                      double *omega) {
  const int ns = cp->ns;
  for (long q = 0; q < n; q++) {
    RateState s;
    ratestate(*cp, s, rho[q], [&](int k) { return Y[q * ns + k]; }, T[q]);
    production(*cp, s, omega + q * ns);
  }
  return 0;
}

// g / Ru T of every species at n temperatures, ln T by tlog
int oracle_gibbs(const OCase *cp, long n, const double *T, double *gRT) {
  for (long q = 0; q < n; q++)
    for (int k = 0; k < cp->ns; k++) gRT[q * cp->ns + k] = gRTspecies(*cp->mech, k, tlog(T[q]), 1.0 / T[q]);
  return 0;
}

int oracle_tlog(long n, const double *x, double *y) {
  for (long q = 0; q < n; q++) y[q] = tlog(x[q]);
  return 0;
}

int oracle_texp(long n, const double *x, double *y) {
  for (long q = 0; q < n; q++) y[q] = texp(x[q]);
  return 0;
}

// the tables tlog and texp read, for a check against the reference's
int oracle_mathtables(double *logtab, double *rcptab, double *exptab, double *scalars) {
  const MathTables &t = mtab();
  std::memcpy(logtab, t.logtab, sizeof t.logtab);
  std::memcpy(rcptab, t.rcptab, sizeof t.rcptab);
  std::memcpy(exptab, t.exptab, sizeof t.exptab);
  scalars[0] = O_LN2, scalars[1] = O_EXPK, scalars[2] = O_LN2BINS_HI, scalars[3] = O_LN2BINS_LO;
  return 0;
}

// cp and h of a pure species n at n temperatures by ideal_cph, per mass
int oracle_species_cph(const OCase *cp, int sp, long n, const double *T, double *cpo, double *ho) {
  const OCase &c = *cp;
  for (long q = 0; q < n; q++) {
    Mom mom = mixmom(c, [&](int k) { return k == sp ? 1.0 : 0.0; });
    ideal_cph(c, mom, T[q], cpo[q], ho[q]);
  }
  return 0;
}

// the state of n cells from Q rows, each from its guess
int oracle_fromQ(const OCase *cp, long n, const double *Q, const double *Tguess, double *state) {
  const int ne = 4 + cp->ns;
  for (long q = 0; q < n; q++) {
    const State st = fromQ(*cp, Q + q * ne, Tguess[q]);
    std::memcpy(state + q * 8, &st, sizeof st);
  }
  return 0;
}

// One stage's combine (peregrine/integrators/kernels/combine.mako:1-13) on a
// block's interior: out = wout out + sum_n w_n X_n, dt on the last term when
// step is set, summed left to right as the rendered expression is.  own says
// whether wout out is a term at all.
int oracle_combine(int nx, int ny, int nz, int ng, int ne, double *out, int own, double wout,
                   int nterms, const double *const *X, const double *w, int step, double dt) {
  const Dims d{nx + 2 * ng, ny + 2 * ng, nz + 2 * ng};
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = ng; i < ng + nx; i++)
    for (int j = ng; j < ng + ny; j++)
      for (int k = ng; k < ng + nz; k++) {
        const long at = d.at(i, j, k) * ne;
        for (int l = 0; l < ne; l++) {
          auto term = [&](int n) {
            return (step && n == nterms - 1) ? w[n] * dt * X[n][at + l] : w[n] * X[n][at + l];
          };
          double acc;
          int n0;
          if (own) {
            acc = wout * out[at + l];
            n0 = 0;
          } else {
            acc = term(0);
            n0 = 1;
          }
          for (int n = n0; n < nterms; n++) acc = acc + term(n);
          out[at + l] = acc;
        }
      }
  return 0;
}

}  // extern "C"

// the threads the oracle's loops share: one for the small cases a test
// runs (a fork per loop costs more than the loop), the host's cores for
// the large ones
extern "C" int oracle_set_threads(int n) {
  omp_set_num_threads(n < 1 ? 1 : n);
  return 0;
}

// register Q's halo of every block filled across the interfaces, a
// rotational periodic's vectors turned (the reference's exchange of a bank)
extern "C" int oracle_exchange(const OCase *cp, OBlock *blocks, int nblocks, const OHaloEntry *map, long nmap) {
  std::vector<OBlock> blks(blocks, blocks + nblocks);
  std::vector<Scratch> scr(nblocks);
  halo_fill(*cp, blks, map, nmap, 1 << 30, 4 + cp->ns, 1, [](OBlock &b, std::vector<Scratch> &, int) { return b.Q; },
            scr);
  return 0;
}
