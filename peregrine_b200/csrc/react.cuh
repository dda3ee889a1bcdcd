// The fused passes: one right-hand side and Runge-Kutta stage of the general
// gas (one to twelve species, calorically or thermally perfect, any flux
// function and reconstruction, inviscid or viscous, coupled chemistry) in
// six to eight launches over every block instead of the per-block path's
// fourteen:
//
//   k_rcell   per cell, halo included: fromQ (the eos's Newton from the
//             cell's last T), then the transport properties and species
//             enthalpies (the per-block path's k_fromQ then k_transport, one
//             thread doing both on the state it just formed)
//             (peregrine/simulator/euler/kernels/state/fromQ.mako:5-19,
//              peregrine/simulator/navstokes/kernels/transport.mako:5-35);
//   k_source  the coupled chemistry source beginning dQ, as on the per-block
//             path (peregrine/simulator/chemint/kernels/source.mako:3-10);
//   k_grads   the cell gradients, then their first halo layer;
//   k_rface   per axis, one face a thread: the advective flux and the
//             diffusive rows in the same thread, stored once (the per-block
//             path stores the advective flux, then reads and stores it again
//             with the diffusive rows added);
//   k_rapply  per cell: the divergence added to the source and the stage's
//             combines, with dQ kept in the thread and never stored
//             (peregrine/simulator/advec/kernels/applyflux.mako:2-11,
//              peregrine/integrators/kernels/combine.mako:1-13).
//
// Each face and cell runs the per-block kernels' own device functions in the
// same order; the two paths' results agree to the rounding of the multiply-
// adds the compiler contracts differently in the two kernels.
//
// Measured and set aside: (a) the chemistry source in the cell kernel, the
// rate state then spilling to local memory, 0.80 ms a pass at 96^3 against
// 0.52 ms for the three passes apart; (b) one tile kernel of every face of a
// plane marching up k with the face fluxes in shared memory and the cell
// records read through L1: at 252 registers a face, one CTA of eight warps
// an SM could not hide the face's two hundred global loads, 4.6 ms a stage
// against 1.0 ms for the three face passes; (c) the three axes' faces in one
// launch ordered slab by slab, so a slab's cell records are read by all its
// faces while in L2: 5.3 to 5.8 ms an RK3 step over slabs of 2 to 96 planes
// against 5.4 ms for the passes per axis (the face passes wait on load
// latency, not on DRAM bandwidth).
#pragma once
#include "chem.cuh"
#include "layout.cuh"
#include "physics.cuh"
#include "plain.cuh"
#include "plain_api.h"

namespace pgb {

// fromQ and the transport of one cell (k_fromQ then k_transport); t over the
// block's full extents, or, with INNER, over its interior cells (a halo
// cell's values are then its source's, copied after)
template <int NS, bool VISC, bool INNER = false>
__global__ void __launch_bounds__(256) k_rcell(const BlockDev *__restrict__ blks, int b,
                                               const double *__restrict__ Qall, double *__restrict__ stall,
                                               double *__restrict__ trall, double *__restrict__ hall,
                                               const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS;
  PGB_WHERE(B, tt);
  long long t = tt;
  if (INNER) {
    if (tt >= (long long)B.nx * B.ny * B.nz) return;
    const int i = (int)(tt % B.nx) + NG, j = (int)((tt / B.nx) % B.ny) + NG;
    const int k = (int)(tt / ((long long)B.nx * B.ny)) + NG;
    t = cell_index(B, i, j, k);
  } else if (t >= B.vol) {
    return;
  }
  const long long v = B.vol;
  const double *Q = Qall + NE * B.cv + t;
  double *st = stall + SW * B.cv + t;
  auto Qf = [&](int c) { return Q[c * v]; };
  const State s = fromQ<NS>(Qf, st[1 * v]);
  st[0 * v] = s.p, st[1 * v] = s.T, st[2 * v] = s.rhoinv, st[3 * v] = s.rho;
  st[4 * v] = s.e, st[5 * v] = s.cp, st[6 * v] = s.gamma, st[7 * v] = s.c;
  if (VISC) {
    double tr[2 + NS], h[NS];
    transport<NS, decltype(Qf), false>(Qf, s, tr, h, 0.0);
    double *trp = trall + (2 + NS) * B.cv + t;
    double *hp = hall + NS * B.cv + t;
#pragma unroll
    for (int n = 0; n < 2 + NS; n++) trp[n * v] = tr[n];
#pragma unroll
    for (int n = 0; n < NS; n++) hp[n * v] = h[n];
  }
}

// what the divergence-and-combine pass reads: dQ (the coupled source on the
// way in, and dQ out when write_dq), the step size and the stage's combines
struct RApplyArgs {
  double *dQ;
  const double *dt;
  int chem;      // 1: dQ holds the source the divergence adds to
  int write_dq;  // 1: store dQ (the right-hand side alone)
  int ncomb;
  RCombine comb[2];
};

// the face of axis A whose high-side cell is R: the advective flux (kepaec on
// the cells as they are, or a Riemann solver FN on the cells or MUSCL's
// sides), then with VISC the diffusive rows added, into F[NE]
template <int NS, int A, int FN, bool VISC>
__device__ __forceinline__ void rface(const BlockDev &B, const double *Q, const double *st, const double *tr,
                                      const double *hs, const double *gr, const double *M, const int lim,
                                      const long long R, double *F) {
  if (FN == 0) advflux_face<NS, A>(B, Q, st, M, R, F);
  else riemann_face<NS, A, FN, false, false>(B, Q, st, M, lim, R, F);
  if (VISC) {
    // the diffusive rows' loads (two cells' gradients, transport and
    // enthalpies) are not hoisted above the advective flux: in flight all at
    // once they would hold twice the registers
    asm volatile("" ::: "memory");
    diffflux_face<NS, A>(B, Q, st, tr, hs, gr, M, R, F);
  }
}

// One face a thread over a pass's faces of axis A: the advective flux and,
// with VISC, the diffusive rows in the same thread, stored once (the
// per-block path's k_riemann then k_diffflux, without the flux's round trip
// between them)
template <int NS, int A, int FN, bool VISC>
__global__ void __launch_bounds__(256, 2) k_rface(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                                               const double *__restrict__ stall, const double *__restrict__ trall,
                                               const double *__restrict__ hall, const double *__restrict__ gall,
                                               const double *__restrict__ met, double *__restrict__ Fall, const int lim,
                                               const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS, NGRAD = NE - 1;
  PGB_WHERE(B, t);
  int i, j, k;
  if (!face_at<A>(B, t, i, j, k)) return;
  const long long R = cell_index(B, i, j, k);
  double F[NE];
  rface<NS, A, FN, VISC>(B, Qall + NE * B.cv, stall + SW * B.cv, VISC ? trall + (2 + NS) * B.cv : nullptr,
                         VISC ? hall + NS * B.cv : nullptr, VISC ? gall + 3 * NGRAD * B.cv : nullptr,
                         met + M_NCOMP * B.cv, lim, R, F);
  double *Fo = Fall + NE * B.cv + R;
#pragma unroll
  for (int l = 0; l < NE; l++) Fo[l * B.vol] = F[l];
}

// The divergence of each interior cell added to its source (the per-block
// applyflux's order) and the stage's combines, dQ kept in the thread
template <int NS>
__global__ void __launch_bounds__(256) k_rapply(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Fi,
                                                const double *__restrict__ Fj, const double *__restrict__ Fk,
                                                const double *__restrict__ met, const RApplyArgs a,
                                                const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS;
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k), v = B.vol;
  const long long sJ = B.X, sK = (long long)B.X * B.Y;
  const double detJinv = met[M_NCOMP * B.cv + M_DETJINV * v + c];
  const double *fi = Fi + NE * B.cv + c, *fj = Fj + NE * B.cv + c, *fk = Fk + NE * B.cv + c;
  const long long at = NE * B.cv + c;
  const double dt = *a.dt;
  double first[NE];
#pragma unroll
  for (int l = 0; l < NE; l++) {
    const double f = (fi[l * v] + fj[l * v] + fk[l * v] - fi[l * v + 1] - fj[l * v + sJ] - fk[l * v + sK]) * detJinv;
    const double dq = a.chem ? a.dQ[at + l * v] + f : f;
    if (a.write_dq) a.dQ[at + l * v] = dq;
    for (int m = 0; m < a.ncomb; m++) {
      const RCombine &cb = a.comb[m];
      auto val = [&](int n) {
        const int s = cb.src[n];
        return s == -1 ? dq : s == -2 ? first[l] : cb.X[n][at + l * v];
      };
      auto term = [&](int n) {
        return (cb.step && n == cb.nterms - 1) ? cb.w[n] * dt * val(n) : cb.w[n] * val(n);
      };
      double acc = term(0);
      for (int n = 1; n < cb.nterms; n++) acc = acc + term(n);
      if (m == 0) first[l] = acc;
      if (cb.write) cb.out[at + l * v] = acc;
    }
  }
}

// The double flux's stage for an inviscid gas with kepaec, a cell a thread:
// its six faces' two-point fluxes (each face formed by both cells it joins;
// kepaec reads the two cells alone), the divergence in the per-block
// applyflux_df's order (the energy row takes the second energy row on the
// cell's low faces, where it is the right cell, the first on its high
// faces), and the stage's combines
// (peregrine/simulator/eulerdf/kernels/flux/function/kepaec.mako:1-21,
//  peregrine/simulator/eulerdf/kernels/applyflux.mako:2-14)
template <int NS>
__global__ void __launch_bounds__(256) k_rcellflux_df(const BlockDev *__restrict__ blks, int b,
                                                      const double *__restrict__ Qall,
                                                      const double *__restrict__ stall,
                                                      const double *__restrict__ met, const RApplyArgs a,
                                                      const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS, NF = NE + 1;
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k), v = B.vol;
  const long long sJ = B.X, sK = (long long)B.X * B.Y;
  const double *Q = Qall + NE * B.cv, *st = stall + SW * B.cv, *M = met + M_NCOMP * B.cv;
  // the six faces one after another, each summed in as it is formed, in
  // the divergence's order (low i, j, k faces added, high ones taken off):
  // one face's rows live at a time
  double acc[NE];
  {
    double f[NF];
    advflux_df_face<NS, 0>(B, Q, st, M, c, f);
#pragma unroll
    for (int l = 0; l < NE; l++) acc[l] = f[l == 4 ? NE : l];
  }
  {
    double f[NF];
    advflux_df_face<NS, 1>(B, Q, st, M, c, f);
#pragma unroll
    for (int l = 0; l < NE; l++) acc[l] = acc[l] + f[l == 4 ? NE : l];
  }
  {
    double f[NF];
    advflux_df_face<NS, 2>(B, Q, st, M, c, f);
#pragma unroll
    for (int l = 0; l < NE; l++) acc[l] = acc[l] + f[l == 4 ? NE : l];
  }
  {
    double f[NF];
    advflux_df_face<NS, 0>(B, Q, st, M, c + 1, f);
#pragma unroll
    for (int l = 0; l < NE; l++) acc[l] = acc[l] - f[l];
  }
  {
    double f[NF];
    advflux_df_face<NS, 1>(B, Q, st, M, c + sJ, f);
#pragma unroll
    for (int l = 0; l < NE; l++) acc[l] = acc[l] - f[l];
  }
  {
    double f[NF];
    advflux_df_face<NS, 2>(B, Q, st, M, c + sK, f);
#pragma unroll
    for (int l = 0; l < NE; l++) acc[l] = acc[l] - f[l];
  }
  const double detJinv = M[M_DETJINV * v + c];
  const long long at = NE * B.cv + c;
  const double dt = *a.dt;
  double first[NE];
#pragma unroll
  for (int l = 0; l < NE; l++) {
    const double dq = acc[l] * detJinv;
    if (a.write_dq) a.dQ[at + l * v] = dq;
    for (int m = 0; m < a.ncomb; m++) {
      const RCombine &cb = a.comb[m];
      auto val = [&](int n) {
        const int s = cb.src[n];
        return s == -1 ? dq : s == -2 ? first[l] : cb.X[n][at + l * v];
      };
      auto term = [&](int n) {
        return (cb.step && n == cb.nterms - 1) ? cb.w[n] * dt * val(n) : cb.w[n] * val(n);
      };
      double acc = term(0);
      for (int n = 1; n < cb.nterms; n++) acc = acc + term(n);
      if (m == 0) first[l] = acc;
      if (cb.write) cb.out[at + l * v] = acc;
    }
  }
}

// Closed constant-volume reactors, a cell each, for the serving pool: a
// uniform closed box has no flux divergence, so a reactor's stage is fromQ
// (the Newton from its last T), the finite-rate source and the stage's
// combines, in one thread (the reference's auto-ignition case, a closed
// box of Euler and chemistry, examples/autoIgnition.py:33-56; the coupled
// source, peregrine/simulator/chemint/kernels/source.mako:3-10).  A
// reactor's registers hold it at row r of a [component][capacity] table.
template <int NS>
__global__ void __launch_bounds__(256) k_reactors(const ReactorStage a) {
  constexpr int NE = 4 + NS;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n) return;
  const long long r = a.rows[t], cap = a.cap;
  auto Qf = [&](int c) { return a.Q[c * cap + r]; };
  const State s = fromQ<NS>(Qf, a.T[r]);
  a.T[r] = s.T;
  double omega[NS];
  cellrates<NS>(Qf, s.T, omega);
  const double dt = *a.dt;
  double first[NE];
#pragma unroll
  for (int l = 0; l < NE; l++) {
    const double dq = l < 5 ? 0.0 : omega[l - 5];
    const long long at = l * cap + r;
    for (int m = 0; m < a.ncomb; m++) {
      const RCombine &cb = a.comb[m];
      auto val = [&](int n) {
        const int src = cb.src[n];
        return src == -1 ? dq : src == -2 ? first[l] : cb.X[n][at];
      };
      auto term = [&](int n) {
        return (cb.step && n == cb.nterms - 1) ? cb.w[n] * dt * val(n) : cb.w[n] * val(n);
      };
      double acc = term(0);
      for (int n = 1; n < cb.nterms; n++) acc = acc + term(n);
      if (m == 0) first[l] = acc;
      if (cb.write) cb.out[at] = acc;
    }
  }
}

// A warp per reactor: every lane forms the same clipped mass fractions, state
// and rate state; the lanes take the reactions' rates of progress k, k + 32,
// ... (the mechanism's global copy, lanes reading different reactions),
// staged in shared memory; then every lane sums the fold in reaction order,
// as cellrates' fold does (the same products and sums in the same order: the
// same bits), and lane l writes component l's combines.
template <int NS>
__global__ void __launch_bounds__(256) k_reactors_warp(const ReactorStage a) {
  constexpr int NE = 4 + NS;
  __shared__ double sh[8][MAXRXN];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * 8 + w;
  if (t >= a.n) return;  // a warp's lanes alike
  const long long r = a.rows[t], cap = a.cap;
  auto Qf = [&](int c) { return a.Q[c * cap + r]; };
  const State st = fromQ<NS>(Qf, a.T[r]);
  // cellrates: the clipped mass fractions and the rate state
  const double rho = Qf(0), rhoinv = 1.0 / rho;
  double Ylast = 1.0, Ysum = 0.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double Yn = fmax(fmin(Qf(5 + n) * rhoinv, 1.0), 0.0);
    Ylast -= Yn;
    Ysum += Yn;
  }
  const double Yscale = 1.0 / fmax(Ysum, 1.0);
  Ylast = fmax(Ylast, 0.0);
  auto Y = [&](int n) { return n < NS - 1 ? fmax(fmin(Qf(5 + n) * rhoinv, 1.0), 0.0) * Yscale : Ylast; };
  RateState<NS> s;
  ratestate<NS>(s, rho, Y, st.T);
  const int nr = kMech.nr;
  for (int k = lane; k < nr; k += 32) {
    const Rxn &rx = gMech.rxn[k];
    double fwd, rev;
    oneway<NS>(rx, s, fwd, rev);
    sh[w][k] = rx.reversible ? fwd - rev : fwd;
  }
  __syncwarp();
  double omega[NS];
#pragma unroll
  for (int n = 0; n < NS; n++) omega[n] = 0.0;
  for (int k = 0; k < nr; k++) {
    const Rxn &rx = kMech.rxn[k];
    const double rp = sh[w][k];
    for (int j = 0; j < rx.nnet; j++) omega[rx.netsp[j]] += rx.netnuMW[j] * rp;
  }
  // every lane has read T above; one writes the new guess
  if (lane == 0) a.T[r] = st.T;
  if (lane >= NE) return;
  const int l = lane;
  const double dt = *a.dt;
  double dq = 0.0;
#pragma unroll
  for (int n = 0; n < NS; n++)
    if (l == 5 + n) dq = omega[n];
  const long long at = l * cap + r;
  double first = 0.0;
  for (int m = 0; m < a.ncomb; m++) {
    const RCombine &cb = a.comb[m];
    auto val = [&](int n) {
      const int src = cb.src[n];
      return src == -1 ? dq : src == -2 ? first : cb.X[n][at];
    };
    auto term = [&](int n) { return (cb.step && n == cb.nterms - 1) ? cb.w[n] * dt * val(n) : cb.w[n] * val(n); };
    double acc = term(0);
    for (int n = 1; n < cb.nterms; n++) acc = acc + term(n);
    if (m == 0) first = acc;
    if (cb.write) cb.out[at] = acc;
  }
}

// a reactor's Q and starting T from its primitives p, u, v, w, T, Y...
// (the reference's fromprims, peregrine/simulator/euler/kernels/state/fromprims.mako)
template <int NS>
__global__ void k_reactor_prims(const double *__restrict__ prims, double *__restrict__ Q, double *__restrict__ T,
                                const int row, const long long cap) {
  constexpr int NE = 4 + NS;
  double q[NE], Qc[NE];
#pragma unroll
  for (int l = 0; l < NE; l++) q[l] = prims[l];
  const State th = fromprims<NS>(q, Qc);
#pragma unroll
  for (int l = 0; l < NE; l++) Q[l * cap + row] = Qc[l];
  T[row] = th.T;
}

}  // namespace pgb
