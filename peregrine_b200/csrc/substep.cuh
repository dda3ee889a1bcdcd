// The sub-stepped chemistry integrator on the per-block path: each cell's
// species and temperature advanced over the step by explicit substeps sized
// to the limiting species' way to its bound, with an equilibrium exit that
// relaxes a settled cell in one move; the mean rate over the step begins dQ
// (peregrine/simulator/chemint/substepped.py:11-68,
//  peregrine/simulator/chemint/kernels/{bulk,stiff,substep,reset}.mako).
//
// Compaction: the bulk pass gives every cell up to bulk-substeps substeps;
// a cell still short of the step's end is listed, in the bin of its count at
// the last right-hand side, and left.  The stiff pass then restarts each
// listed cell from the start with the cap, so its result is the one-pass
// form's; it is one persistent launch whose warps take the list 32 cells at
// a time, the bins of the most substeps first, so the longest cells start
// first and a warp's lanes take about as many substeps each.
#pragma once
#include "chem.cuh"
#include "layout.cuh"
#include "physics.cuh"

namespace pgb {

// cp / R of species n in ln T (peregrine/simulator/mixture/eos/kernels/species.mako:3-7)
__device__ __forceinline__ double cpRspecies(const int n, const double u) {
  double cpR = 0.0;
#pragma unroll
  for (int m = MAXT - 1; m >= 0; m--)
    if (m < kSp.ncppoly) cpR = cpR * u + kSp.cppoly[n * MAXT + m];
  return cpR;
}

// the internal energy per mass of species n (species.mako:9-14, 23-27)
__device__ __forceinline__ double especies(const int n, const double T, const double u, const double Tinv) {
  double hRT = 0.0;
#pragma unroll
  for (int m = MAXT - 1; m >= 0; m--)
    if (m < kSp.nh) hRT = hRT * u + kSp.hpoly[n * MAXT + m];
  hRT += kSp.h298[n] * Tinv;
  return (hRT - 1.0) * T * kSp.Rsp[n];
}

// integrate (substep.mako:4-87): up to limit substeps from Y, T over what
// remains of the step; src gathers the mean rate; EXIT judges the
// equilibrium exit at the first substep.  With WARP a whole warp integrates
// the one cell, its lanes over the reactions (every lane holds the cell's
// state alike).  Returns the substeps taken.
template <int NS, bool EXIT, bool WARP = false>
__device__ int substep_integrate(const double rho, const double rhoinv, const double step, double *Y, double &T,
                                 double *src, double &remaining, const int limit, const double eqtol,
                                 const double stepfrac, const int lane = 0) {
  const double eps = 2.220446049250313e-16, tiny = 2.2250738585072014e-308, stepinv = 1.0 / step;
  auto Yof = [&](int n) { return Y[n]; };
  double rate[NS];
  int sub = 0;
  bool early = false;
  for (; sub < limit && remaining > stepfrac; sub++) {
    RateState<NS> s;
    ratestate<NS>(s, rho, Yof, T);
    // the first substep's fold carries the destruction rates the exit relaxes by
    double D[NS];
    if (WARP)
      fold_warp<NS>(s, rate, lane);
    else if (EXIT && eqtol > 0.0 && sub == 0)
      fold<NS, true>(s, rate, D);
    else
      fold<NS, false>(s, rate, nullptr);
    // the limiting species by cross-multiplying, one quotient at the end
    double abest = 0.0, bbest = 0.0;
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const double sign = copysign(1.0, rate[n]);
      const double headroom = 0.5 * ((1.0 - sign) * Y[n] + (1.0 + sign) * (1.0 - Y[n]));
      const double a = rho * fmax(headroom, eps), b = fmax(fabs(rate[n]), tiny);
      if (n == 0 || a * bbest < abest * b) {
        abest = a;
        bbest = b;
      }
    }
    const double share = fmin(remaining, abest / bbest * stepinv);
    // the temperature's rate at constant volume
    double cv = 0.0, dTdt = 0.0;
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const double cpR = cpRspecies(n, s.logT);
      const double e = especies(n, T, s.logT, s.Tinv);
      cv += (cpR - 1.0) * kSp.Rsp[n] * Y[n];
      dTdt -= e * rate[n];
    }
    const double cvrhoinv = 1.0 / (cv * rho);
    dTdt *= cvrhoinv;
    if (EXIT && eqtol > 0.0) {
      // judged at the first substep only: nothing moves past the tolerance
      // over what remains, so the rest is one move with each species relaxed
      // at its destruction frequency
      const double tleft = remaining * step, tleftinv = 1.0 / tleft;
      bool settled = sub == 0 && tleft > 0.0 && fabs(dTdt) * tleft < 0.1;
#pragma unroll
      for (int n = 0; n < NS; n++) settled = settled && fabs(rate[n] * rhoinv) * tleft < eqtol;
      if (settled) {
        double dT = 0.0;
#pragma unroll
        for (int n = 0; n < NS; n++) {
          const double rhoden = rho * fmax(Y[n], kMech.cfloor * kSp.MW[n] * rhoinv);
          const double move = fmax((rate[n] * rhoinv) * tleft * rhoden / (rhoden + D[n] * tleft), -Y[n]);
          const double r = move * rho * tleftinv;
          const double e = especies(n, T, s.logT, s.Tinv);
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
#pragma unroll
    for (int n = 0; n < NS; n++) {
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

// startstate (substep.mako:89-95): the clipped mass fractions
// (peregrine/simulator/euler/kernels/solution.mako:25-38) and the cell's T
template <int NS, class QF>
__device__ __forceinline__ void substep_start(QF Q, const double rhoinv, double *Y, double *src) {
  double Ylast = 1.0, Ysum = 0.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double Yn = fmax(fmin(Q(5 + n) * rhoinv, 1.0), 0.0);
    Ylast -= Yn;
    Ysum += Yn;
  }
  const double Yscale = 1.0 / fmax(Ysum, 1.0);
  Ylast = fmax(Ylast, 0.0);
#pragma unroll
  for (int n = 0; n < NS; n++) {
    Y[n] = n < NS - 1 ? fmax(fmin(Q(5 + n) * rhoinv, 1.0), 0.0) * Yscale : Ylast;
    src[n] = 0.0;
  }
}

// beginsource (cell.mako:14-19): dQ begins with the mean rates
template <int NS>
__device__ __forceinline__ void substep_source(double *dQ, const long long v, const double *src) {
#pragma unroll
  for (int l = 0; l < 5; l++) dQ[l * v] = 0.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) dQ[(5 + n) * v] = src[n];
}

// the bulk pass (bulk.mako:3-34) over the interior cells
template <int NS>
__global__ void k_substep_bulk(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                               const double *__restrict__ stall, double *__restrict__ dQall, int *__restrict__ subs,
                               const double *__restrict__ dt, SubstepOpts o, StiffList list,
                               const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS;
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k), v = B.vol;
  const double *Q = Qall + NE * B.cv + c;
  auto Qf = [&](int l) { return Q[l * v]; };
  const double rho = Qf(0), rhoinv = 1.0 / rho, step = *dt;
  double Y[NS], src[NS], T = stall[SW * B.cv + 1 * v + c], remaining = 1.0;
  substep_start<NS>(Qf, rhoinv, Y, src);
  int *sub = subs + B.cv + c;
  const int taken =
      substep_integrate<NS, true>(rho, rhoinv, step, Y, T, src, remaining, o.bulk, o.eqtol, o.stepfrac);
  if (o.bulk < o.cap && remaining > o.stepfrac) {
    // binned by the cell's count at the last right-hand side, a cell just
    // turned stiff to the top bin, the ends taking what falls past them
    int bin = 0;
    if (o.bins > 1) {
      const int expected = *sub > o.bulk ? *sub : o.cap;
      const int spaced = (int)(log((double)expected * o.limitinv) * o.binscale);
      bin = spaced < 0 ? 0 : (spaced >= o.bins ? o.bins - 1 : spaced);
    }
    // warp-aggregated: one atomic per bin the warp's listed lanes fall in,
    // one for the total
    const unsigned int lane = threadIdx.x & 31, act = __activemask();
    const unsigned int same = __match_any_sync(act, bin);
    const int leader = __ffs(same) - 1;
    unsigned int slot = 0;
    if ((int)lane == leader) slot = atomicAdd(&list.head[1 + bin], (unsigned int)__popc(same));
    slot = __shfl_sync(same, slot, leader) + __popc(same & ((1u << lane) - 1u));
    if ((int)lane == __ffs(act) - 1) atomicAdd(&list.head[0], (unsigned int)__popc(act));
    list.cells[(long long)bin * list.capacity + slot] = make_int2(where_.x, (int)c);
    return;
  }
  *sub = taken;
  substep_source<NS>(dQall + NE * B.cv + c, v, src);
}

// the stiff pass (stiff.mako:3-18): the listed cells from the start with the
// cap and no exit, the list read top bin first.  A long list goes a cell to
// a lane, the warps taking it 32 cells at a time; a list no longer than two
// cells a warp goes a cell to a warp, its lanes over the reactions, so a few
// cells that take the cap are not one lane's serial substeps
template <int NS>
__global__ void k_substep_stiff(const BlockDev *__restrict__ blks, const double *__restrict__ Qall,
                                const double *__restrict__ stall, double *__restrict__ dQall, int *__restrict__ subs,
                                const double *__restrict__ dt, SubstepOpts o, StiffList list) {
  constexpr int NE = 4 + NS;
  const int lane = threadIdx.x & 31;
  const unsigned int total = list.head[0];
  const unsigned int nwarps = gridDim.x * (blockDim.x >> 5);
  const bool per_warp = total <= 2u * nwarps;
  // position p in the list read top bin first
  auto at = [&](unsigned int p) {
    int bin = o.bins - 1;
    for (; bin > 0; bin--) {
      const unsigned int n = list.head[1 + bin];
      if (p < n) break;
      p -= n;
    }
    return list.cells[(long long)bin * list.capacity + p];
  };
  for (;;) {
    unsigned int base = 0;
    if (lane == 0) base = atomicAdd(&list.head[o.bins + 1], per_warp ? 1u : 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) return;  // the warp's lanes alike
    const unsigned int p = per_warp ? base : base + lane;
    if (p < total) {
      const int2 code = at(p);
      const BlockDev &B = blks[code.x];
      const long long c = code.y, v = B.vol;
      const double *Q = Qall + NE * B.cv + c;
      auto Qf = [&](int l) { return Q[l * v]; };
      const double rho = Qf(0), rhoinv = 1.0 / rho, step = *dt;
      double Y[NS], src[NS], T = stall[SW * B.cv + 1 * v + c], remaining = 1.0;
      substep_start<NS>(Qf, rhoinv, Y, src);
      int taken;
      if (per_warp)
        taken = substep_integrate<NS, false, true>(rho, rhoinv, step, Y, T, src, remaining, o.cap, o.eqtol,
                                                   o.stepfrac, lane);
      else
        taken = substep_integrate<NS, false>(rho, rhoinv, step, Y, T, src, remaining, o.cap, o.eqtol, o.stepfrac);
      if (!per_warp || lane == 0) {
        subs[B.cv + c] = taken;
        substep_source<NS>(dQall + NE * B.cv + c, v, src);
      }
    }
    __syncwarp();
  }
}

}  // namespace pgb
