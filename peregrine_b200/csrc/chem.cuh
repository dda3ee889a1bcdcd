// Finite-rate chemistry on the device: the table log and exp, a cell's rate
// state, the fold over the reactions, and the coupled source that begins dQ.
//
// The mechanism is data, not code: one constant struct holds every
// reaction's columns (its kind, the species and orders of each side, its
// Arrhenius and falloff constants), so one kernel serves any mechanism.  A
// warp's threads walk the reactions in step, so each reaction's constants are
// one broadcast read.  The reference renders the same fold with the species
// indices as literals (peregrine/simulator/mixture/chemistry/kernels/finiterate.mako);
// the arithmetic per reaction is the same, in the same order.
#pragma once
#include "chem_types.h"
#include "layout.cuh"
#include "physics.cuh"

namespace pgb {

static __constant__ Mech kMech;
// the same tables in global memory, for the passes whose lanes read
// different reactions at once (constant memory serialises differing addresses)
static __device__ Mech gMech;

// the table log's and exp's tables, read per lane at differing bins: global
// memory through the read-only cache rather than constant memory, which
// would serialise a warp's differing addresses
static __device__ MathTables gMath;

// tlog: log x as e ln 2 + log m_k + u times a fourth-degree series, u the
// mantissa over its bin's centre less one
// (peregrine/backend/base/kernels/mathfns.mako:6-26)
__device__ __forceinline__ double tlog(const double x) {
  long long bits = __double_as_longlong(x);
  const int expo = (int)((bits >> 52) & 0x7ff) - 1022;
  const int bin = (int)((bits >> 45) & 127);
  bits = (bits & 0x000fffffffffffffLL) | 0x3fe0000000000000LL;
  const double mant = __longlong_as_double(bits);
  const double u = mant * __ldg(&gMath.rcptab[bin]) - 1.0;
  double series = 0.2;
  series = series * u - 0.25;
  series = series * u + 1.0 / 3.0;
  series = series * u - 0.5;
  series = series * u + 1.0;
  return expo * 0x1.62e42fefa39efp-1 + __ldg(&gMath.logtab[bin]) + u * series;
}

// texp: exp x as 2^n 2^(j/64) times a fifth-degree series in the remainder,
// the nearest integer k = 64 n + j found by adding 1.5 2^52
// (peregrine/backend/base/kernels/mathfns.mako:30-53)
__device__ __forceinline__ double texp(const double v) {
  const double t = v * 0x1.71547652b82fep+6 + 6755399441055744.0;
  long long bits = __double_as_longlong(t);
  const int kexp = (int)bits, nexp = kexp >> 6;
  const double kd = t - 6755399441055744.0;
  const double r = (v - kd * 0x1.62e42fef00000p-7) - kd * 0x1.473de6af278edp-40;
  double series = 1.0 / 120.0;
  series = series * r + 1.0 / 24.0;
  series = series * r + 1.0 / 6.0;
  series = series * r + 0.5;
  series = series * r + 1.0;
  series = series * r + 1.0;
  const double m = __ldg(&gMath.exptab[kexp & 63]) * series;
  bits = __double_as_longlong(m);
  bits += (long long)(nexp > -1022 ? nexp : -1022) << 52;
  return __longlong_as_double(bits);
}

// a cell's rate state (finiterate.mako:136-183)
template <int NS>
struct RateState {
  double T, logT, Tinv, logprefRuT, prefRuT, prefRuTinv, ctot;
  double logc[NS], gRT[NS], cG[NS];
  double logtb[MAXTB], ctb[MAXTB];
};

template <int NS, class YF>
__device__ __forceinline__ void ratestate(RateState<NS> &s, const double rho, YF Y, const double T) {
  const Mech &m = kMech;
  s.T = T;
  s.logT = tlog(T);
  s.Tinv = 1.0 / T;
  s.logprefRuT = m.logprefRu - s.logT;
  s.prefRuT = m.prefRu * s.Tinv;
  s.prefRuTinv = m.Rupref * T;
  s.ctot = 0.0;
#pragma unroll
  for (int n = 0; n < NS; n++) {
    const double c = rho * Y(n) * kSp.MWinv[n];
    s.ctot += c;
    // gRTspecies (peregrine/simulator/mixture/eos/kernels/species.mako:17-22)
    double g = 0.0;
#pragma unroll
    for (int t = MAXT; t >= 0; t--)
      if (t < m.ngp) g = g * s.logT + m.gpoly[n][t];
    s.gRT[n] = g + kSp.h298[n] * s.Tinv;
    if (m.logform) s.logc[n] = fmax(m.logcfloor, tlog(c));
    if (m.product) s.cG[n] = fmax(c, 0.0) * texp(s.gRT[n]);
  }
  for (int j = 0; j < m.ntb; j++) {
    double ctbc = m.tbdefeff[j] * s.ctot;
    for (int i = 0; i < m.tbneff[j]; i++) {
      const int sp = m.tbeffsp[j][i];
      ctbc += m.tbeffdev[j][i] * (rho * Y(sp) * kSp.MWinv[sp]);
    }
    s.ctb[j] = ctbc;
    s.logtb[j] = tlog(fmax(2.2250738585072014e-308, ctbc));
  }
}

// Troe's broadening added to ln k (finiterate.mako:48-63)
__device__ __forceinline__ double troeblend(const Rxn &r, const double logT, const double logpr) {
  const Mech &m = kMech;
  double lfc;
  if (r.nfcent == 0) {
    lfc = m.lfcfloor;
  } else {
    const double tf = (logT - m.troeuc) * m.troeuhinv;
    lfc = m.lfcpoly[r.troe][m.nlfc - 1];
    for (int k = m.nlfc - 2; k >= 0; k--) lfc = lfc * tf + m.lfcpoly[r.troe][k];
  }
  const double C = -0.4 - 0.67 * lfc, N = 0.75 - 1.27 * lfc;
  const double A = logpr * 0.4342944819032518 + C, B = N - 0.14 * A, B2 = B * B;
  return lfc * B2 / (B2 + A * A) * 2.302585092994046;
}

// one reaction's one-way rates of progress, fwd and rev (0 for an
// irreversible one): the product form (finiterate.mako:66-125) or the log form
// with the double fold's one-way rates (finiterate.mako:7-46, 201-214)
template <int NS>
__device__ __forceinline__ void oneway(const Rxn &r, const RateState<NS> &s, double &fwd, double &rev) {
  const Mech &m = kMech;
  double lk = r.logA;
  if (r.b != 0.0) lk += r.b * s.logT;
  if (r.EaR != 0.0) lk -= r.EaR * s.Tinv;
  const bool falloff = r.kind >= 2, thirdbody = r.kind != 0;
  double logpr = 0.0;
  if (falloff) {
    logpr = s.logtb[r.tb] + r.logprA;
    if (r.prb != 0.0) logpr += r.prb * s.logT;
    if (r.prEaR != 0.0) logpr -= r.prEaR * s.Tinv;
  }
  if (r.product) {
    double pfac = 0.0;
    if (falloff) {
      const double pr = texp(fmin(logpr, m.expclamp));
      pfac = pr / (1.0 + pr);
    }
    if (r.kind == 3) lk += troeblend(r, s.logT, logpr);
    double xk = lk;
    for (int j = 0; j < r.nreact; j++) xk -= r.reactnu[j] * s.gRT[r.reactsp[j]];
    double K = texp(fmin(xk, m.expclamp));
    if (thirdbody && !falloff) K *= s.ctb[r.tb];
    if (falloff) K *= pfac;
    fwd = K;
    for (int j = 0; j < r.nreact; j++) {
      const double cg = s.cG[r.reactsp[j]];
      for (int q = 0; q < (int)r.reactnu[j]; q++) fwd *= cg;
    }
    rev = 0.0;
    if (r.reversible) {
      rev = K;
      const double f = r.nusum > 0.0 ? s.prefRuTinv : s.prefRuT;
      for (int q = 0; q < (int)fabs(r.nusum); q++) rev *= f;
      for (int j = 0; j < r.nprod; j++) {
        const double cg = s.cG[r.prodsp[j]];
        for (int q = 0; q < (int)r.prodnu[j]; q++) rev *= cg;
      }
    }
    return;
  }
  if (thirdbody && !falloff) lk += s.logtb[r.tb];
  if (falloff) lk += fmin(logpr, 0.0) - log1p(texp(-fabs(logpr)));
  if (r.kind == 3) lk += troeblend(r, s.logT, logpr);
  double lrp = lk;
  for (int j = 0; j < r.nfwd; j++) lrp += r.fwdorder[j] * s.logc[r.fwdsp[j]];
  fwd = texp(fmin(lrp, m.expclamp));
  rev = 0.0;
  if (!r.reversible) return;
  double diff = r.nusum != 0.0 ? r.nusum * s.logprefRuT : 0.0;
  for (int j = 0; j < r.nnet; j++) diff -= r.netnu[j] * (s.gRT[r.netsp[j]] + s.logc[r.netsp[j]]);
  rev = texp(fmin(lrp - diff, m.expclamp));
}

// one reaction's net rate of progress; an irreversible one's is its forward rate
template <int NS>
__device__ __forceinline__ double progress(const Rxn &r, const RateState<NS> &s) {
  double fwd, rev;
  oneway<NS>(r, s, fwd, rev);
  return r.reversible ? fwd - rev : fwd;
}

// the fold: the net production rates omega and, with D, the destruction
// rates, kg / m^3 / s, in one pass over the reactions (finiterate.mako:186-236)
template <int NS, bool WITHD>
__device__ __forceinline__ void fold(const RateState<NS> &s, double *omega, double *D) {
#pragma unroll
  for (int n = 0; n < NS; n++) omega[n] = 0.0;
  if (WITHD)
#pragma unroll
    for (int n = 0; n < NS; n++) D[n] = 0.0;
  for (int k = 0; k < kMech.nr; k++) {
    const Rxn &r = kMech.rxn[k];
    double fwd, rev;
    oneway<NS>(r, s, fwd, rev);
    const double rp = r.reversible ? fwd - rev : fwd;
    for (int j = 0; j < r.nnet; j++) {
      const double nuMW = r.netnuMW[j];
      omega[r.netsp[j]] += nuMW * rp;
      // a species a side destroys: the forward rate where it is a reactant, the reverse where a product
      if (WITHD) D[r.netsp[j]] += (nuMW < 0.0 ? -nuMW : 0.0) * fwd + (nuMW > 0.0 ? nuMW : 0.0) * rev;
    }
  }
}

// the fold with the reactions across a warp's lanes, each lane its own
// reactions' terms per species, a butterfly sum after: every lane ends with
// the same omega (the terms' order differs from the one-lane fold's)
template <int NS>
__device__ __forceinline__ void fold_warp(const RateState<NS> &s, double *omega, const int lane) {
  double part[NS];
#pragma unroll
  for (int n = 0; n < NS; n++) part[n] = 0.0;
  const int nr = kMech.nr;
  for (int k = lane; k < nr; k += 32) {
    const Rxn &r = gMech.rxn[k];
    double fwd, rev;
    oneway<NS>(r, s, fwd, rev);
    const double rp = r.reversible ? fwd - rev : fwd;
    for (int j = 0; j < r.nnet; j++) {
      const double add = r.netnuMW[j] * rp;
      const int sp = r.netsp[j];
#pragma unroll
      for (int n = 0; n < NS; n++)
        if (sp == n) part[n] += add;
    }
  }
#pragma unroll
  for (int n = 0; n < NS; n++) {
    double x = part[n];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    omega[n] = x;
  }
}

// cellrates: the clipped mass fractions (peregrine/simulator/euler/kernels/solution.mako:25-38),
// the rate state at the cell's T and the net production rates, kg / m^3 / s
// (peregrine/simulator/chemint/kernels/cell.mako:5-12, finiterate.mako:186-231)
template <int NS, class QF>
__device__ __forceinline__ void cellrates(QF Q, const double T, double *omega) {
  const double rho = Q(0), rhoinv = 1.0 / rho;
  double Ylast = 1.0, Ysum = 0.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double Yn = fmax(fmin(Q(5 + n) * rhoinv, 1.0), 0.0);
    Ylast -= Yn;
    Ysum += Yn;
  }
  const double Yscale = 1.0 / fmax(Ysum, 1.0);
  Ylast = fmax(Ylast, 0.0);
  auto Y = [&](int n) { return n < NS - 1 ? fmax(fmin(Q(5 + n) * rhoinv, 1.0), 0.0) * Yscale : Ylast; };
  RateState<NS> s;
  ratestate<NS>(s, rho, Y, T);
  fold<NS, false>(s, omega, nullptr);
}

// the coupled source: dQ begins with zeros in the mass, momentum and energy
// rows and the carried species' production rates in theirs; the fluxes add to
// it (peregrine/simulator/chemint/kernels/source.mako:3-10, cell.mako:14-19)
template <int NS>
__global__ void k_source(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                         const double *__restrict__ stall, double *__restrict__ dQall,
                         const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS;
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k), v = B.vol;
  const double *Q = Qall + NE * B.cv + c;
  const double T = stall[SW * B.cv + 1 * v + c];
  double omega[NS];
  cellrates<NS>([&](int l) { return Q[l * v]; }, T, omega);
  double *dQ = dQall + NE * B.cv + c;
#pragma unroll
  for (int l = 0; l < 5; l++) dQ[l * v] = 0.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) dQ[(5 + n) * v] = omega[n];
}

// the production rates of independent states (rho, Y of every species, T),
// as the kernels form them, without the clipping: a check of the fold alone
template <int NS>
__global__ void k_production(long long n, const double *__restrict__ rho, const double *__restrict__ Y,
                             const double *__restrict__ T, double *__restrict__ omega) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= n) return;
  RateState<NS> s;
  ratestate<NS>(s, rho[q], [&](int k) { return Y[q * NS + k]; }, T[q]);
  double w[NS];
  fold<NS, false>(s, w, nullptr);
#pragma unroll
  for (int k = 0; k < NS; k++) omega[q * NS + k] = w[k];
}

}  // namespace pgb
