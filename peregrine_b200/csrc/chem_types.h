// The finite-rate mechanism's tables as the device reads them, and the
// tables of the table log and exp: plain structs the host fills, shared by
// the library's translation units.
#pragma once
#include <cmath>

#include "physics.cuh"

namespace pgb {

constexpr int MAXRXN = 64, MAXTB = 8, MAXTROE = 8, MAXLFC = 16, MAXSIDE = 4, MAXNET = 8;

// one reaction (the columns of FiniteRateModel.rxnconsts,
// peregrine/simulator/mixture/chemistry/finiterate.py:122-160)
struct Rxn {
  int kind;  // 0 elementary, 1 three-body, 2 Lindemann falloff, 3 Troe falloff
  int reversible, product, tb, troe, nfcent;
  int nfwd, nreact, nprod, nnet;
  int fwdsp[MAXSIDE], reactsp[MAXSIDE], prodsp[MAXSIDE], netsp[MAXNET];
  double fwdorder[MAXSIDE], reactnu[MAXSIDE], prodnu[MAXSIDE], netnu[MAXNET], netnuMW[MAXNET];
  double logA, b, EaR, logprA, prb, prEaR, nusum;
};

struct Mech {
  int nr, ntb, nlfc, ngp;  // reactions, third-body sets, Troe fit terms, Gibbs fit terms
  int logform, product;  // whether any reaction takes the log form / the product form
  double logprefRu, prefRu, Rupref, logcfloor, troeuc, troeuhinv;
  double cfloor;    // exp(logcfloor): the concentration floor of the equilibrium exit's relaxation
  double expclamp;  // ln(DBL_MAX) - ln(2 maxgain): the largest ln rate whose production rates stay finite
  double lfcfloor;  // log10 of the smallest normal double, a Troe centre without terms
  double tbdefeff[MAXTB];
  int tbneff[MAXTB];
  int tbeffsp[MAXTB][MAXNS];
  double tbeffdev[MAXTB][MAXNS];
  double lfcpoly[MAXTROE][MAXLFC];
  double gpoly[MAXNS][MAXT + 1];  // g / Ru T in ln T less h298 / T, one more term than cp
  Rxn rxn[MAXRXN];
};

// the sub-stepped chemistry's options (peregrine/simulator/chemint/substepped.py:14-19, 47-52)
struct SubstepOpts {
  int cap, bulk, bins;
  double eqtol, stepfrac;
  double limitinv, binscale;  // the bulk pass's 1 / limit and bins / ln(cap / limit)
};

// the stiff list: head[0] every listed cell, head[1 + b] bin b's count,
// head[bins + 1] the stiff pass's work counter; bin b's codes from cell
// b * capacity
struct StiffList {
  unsigned int *head;
  int2 *cells;  // (block, cell index in the block's full layout)
  long long capacity;
};

// the table log's and exp's tables
struct MathTables {
  double logtab[128], rcptab[128], exptab[64];
};

// the tables by the reference's definitions (peregrine/backend/base/mathfns.py:1-22):
// bin centres of the mantissa in [0.5, 1), their logs and reciprocals, and
// the 64 fractional powers of two
inline void math_tables_fill(MathTables &t) {
  for (int k = 0; k < 128; k++) {
    const double m = 0.5 + (k + 0.5) / (2 * 128);
    t.logtab[k] = std::log(m);
    t.rcptab[k] = 1.0 / m;
  }
  for (int j = 0; j < 64; j++) t.exptab[j] = std::pow(2.0, j / 64.0);
}

}  // namespace pgb
