// The plain per-block path: the reference's kernels one by one, one launch
// per block and kernel, each pass a round trip through HBM as in the
// reference's rhs graph (peregrine/simulator/advec/simulator.py:57-87,
// peregrine/simulator/advecdiff/simulator.py:110-124).  It is the baseline
// the fused path is measured against and the path for physics the fused
// kernel does not take.  Every kernel's block is blks[b + blockIdx.y]: a
// launch of one block has gridDim.y 1, a packed launch covers many blocks
// at once, one grid row each (the serving pool's).
#pragma once
#include "layout.cuh"
#include "physics.cuh"

namespace pgb {

// a vector of three components at stride st turned by R
__device__ __forceinline__ void rotate3(double *x, const long long st, const double *R) {
  const double a = x[0], b = x[st], c = x[2 * st];
  x[0] = R[0] * a + R[1] * b + R[2] * c;
  x[st] = R[3] * a + R[4] * b + R[5] * c;
  x[2 * st] = R[6] * a + R[7] * b + R[8] * c;
}

// the halo fill over every block at once: comps components per entry, the
// vectors an entry's rotation turns given by vec (a component, or
// HALO_TENSOR for the gradients), rots the case's rotations, 3 x 3 each
// (the reference's place kernel, peregrine/multiblock/collections/exchange/kernels/place.mako:3-36)
// one halo cell: C components (comps of them when C is 0) copied from the
// source cell, then the vectors its rotation turns.  A source is an interior
// cell, which no thread of the fill writes, so all of a chunk's components
// are loaded (read-only path) before any is stored: the loads are in flight
// together, not one round trip each.
template <int C, bool ROT = true>
__device__ __forceinline__ void halo_copy(double *__restrict__ base, const int comps, const int vec,
                                          const double *__restrict__ rots, const long long dcv, const int didx,
                                          const int dvol, const long long scv, const int sidx, const int svol,
                                          const int rot, const int stride) {
  // a block's array starts stride x its cell offset in (its component
  // count, or more where the first comps of wider records are copied)
  double *d = base + stride * dcv + didx;
  const double *s = base + stride * scv + sidx;
  if constexpr (C > 0) {
    double v[C];
#pragma unroll
    for (int q = 0; q < C; q++) v[q] = __ldg(s + (long long)q * svol);
#pragma unroll
    for (int q = 0; q < C; q++) d[(long long)q * dvol] = v[q];
  } else {
    constexpr int CH = 4;
    for (int c0 = 0; c0 < comps; c0 += CH) {
      double v[CH];
#pragma unroll
      for (int q = 0; q < CH; q++)
        if (c0 + q < comps) v[q] = __ldg(s + (long long)(c0 + q) * svol);
#pragma unroll
      for (int q = 0; q < CH; q++)
        if (c0 + q < comps) d[(long long)(c0 + q) * dvol] = v[q];
    }
  }
  if (ROT && rot && rots && vec != HALO_SCALARS) {
    const double *R = rots + 9 * (rot - 1);
    const long long st = dvol;
    if (vec >= 0) {
      rotate3(d + vec * st, st, R);
    } else {
      // each row's directions, then the velocity rows down every direction
      for (int r = 0; r < comps / 3; r++) rotate3(d + 3 * r * st, st, R);
      for (int m = 0; m < 3; m++) rotate3(d + m * st, 3 * st, R);
    }
  }
}

static __global__ void k_halo(double *__restrict__ base, const HaloEntry *__restrict__ tab, long long n, int comps,
                              int vec = HALO_SCALARS, const double *__restrict__ rots = nullptr, int stride = 0) {
  if (stride == 0) stride = comps;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const HaloEntry h = tab[e];
    halo_copy<0>(base, comps, vec, rots, h.dcv, h.didx, h.dvol, h.scv, h.sidx, h.svol, h.rot, stride);
  }
}

// the same fill over boxes: CTA x (256 threads) fills chunk cta[x].y of box
// cta[x].x, or, where cta[x].x is -1, entries 256 cta[x].y .. of the cells no
// box holds; no per-cell record is read for a box's cells
template <int C, bool ROT>
static __global__ void __launch_bounds__(256) k_halo_boxes(double *__restrict__ base,
                                                           const HaloPatch *__restrict__ boxes,
                                                           const int2 *__restrict__ cta,
                                                           const HaloEntry *__restrict__ rest, long long nrest,
                                                           int comps, int vec = HALO_SCALARS,
                                                           const double *__restrict__ rots = nullptr,
                                                           int stride = 0) {
  if (stride == 0) stride = comps;
  const int2 w = cta[blockIdx.x];
  const int t = w.y * 256 + (int)threadIdx.x;
  if (w.x < 0) {
    if (t >= nrest) return;
    const HaloEntry h = rest[t];
    halo_copy<C, ROT>(base, comps, vec, rots, h.dcv, h.didx, h.dvol, h.scv, h.sidx, h.svol, h.rot, stride);
    return;
  }
  const HaloPatch &p = boxes[w.x];
  if (t >= p.cells) return;
  const int x0 = t % p.n0, r = t / p.n0, x1 = r % p.n1, x2 = r / p.n1;
  const int didx = p.d0 + x0 * p.dst[0] + x1 * p.dst[1] + x2 * p.dst[2];
  const int sidx = p.s0 + x0 * p.sst[0] + x1 * p.sst[1] + x2 * p.sst[2];
  halo_copy<C, ROT>(base, comps, vec, rots, p.dcv, didx, p.dvol, p.scv, sidx, p.svol, p.rot, stride);
}

// two registers' halos in one pass over the boxes: C1 components of the
// first (its vector at vec turned by a cell's rotation), then C2 scalar
// components of the second; each with its own stride (0: its component
// count).  A CTA fills 256 cells of one box, or 256 leftover entries.
template <int C1, int C2, bool ROT>
static __global__ void __launch_bounds__(256) k_halo_boxes2(double *__restrict__ base1, int vec, int stride1,
                                                            double *__restrict__ base2, int stride2,
                                                            const HaloPatch *__restrict__ boxes,
                                                            const int2 *__restrict__ cta,
                                                            const HaloEntry *__restrict__ rest, long long nrest,
                                                            const double *__restrict__ rots) {
  if (stride1 == 0) stride1 = C1;
  if (stride2 == 0) stride2 = C2;
  const int2 w = cta[blockIdx.x];
  const int t = w.y * 256 + (int)threadIdx.x;
  if (w.x < 0) {
    if (t >= nrest) return;
    const HaloEntry h = rest[t];
    halo_copy<C1, ROT>(base1, C1, vec, rots, h.dcv, h.didx, h.dvol, h.scv, h.sidx, h.svol, h.rot, stride1);
    halo_copy<C2, false>(base2, C2, HALO_SCALARS, rots, h.dcv, h.didx, h.dvol, h.scv, h.sidx, h.svol, 0, stride2);
    return;
  }
  const HaloPatch &p = boxes[w.x];
  if (t >= p.cells) return;
  const int x0 = t % p.n0, r = t / p.n0, x1 = r % p.n1, x2 = r / p.n1;
  const int didx = p.d0 + x0 * p.dst[0] + x1 * p.dst[1] + x2 * p.dst[2];
  const int sidx = p.s0 + x0 * p.sst[0] + x1 * p.sst[1] + x2 * p.sst[2];
  halo_copy<C1, ROT>(base1, C1, vec, rots, p.dcv, didx, p.dvol, p.scv, sidx, p.svol, p.rot, stride1);
  halo_copy<C2, false>(base2, C2, HALO_SCALARS, rots, p.dcv, didx, p.dvol, p.scv, sidx, p.svol, 0, stride2);
}

// the box fill of a register of comps components: the kernel built for that
// count where there is one (a stage's Q), else the loop; the rotation code
// only where the case has rotations and the register has vectors
template <bool ROT, int... Cs>
inline void halo_boxes_rot(unsigned grid, cudaStream_t st, double *base, const HaloPatch *boxes, const int2 *cta,
                           const HaloEntry *rest, long long nrest, int comps, int vec, const double *rots,
                           int stride) {
  bool done = false;
  ((!done && comps == Cs
        ? (k_halo_boxes<Cs, ROT><<<grid, 256, 0, st>>>(base, boxes, cta, rest, nrest, comps, vec, rots, stride),
           done = true)
        : false),
   ...);
  if (!done) k_halo_boxes<0, ROT><<<grid, 256, 0, st>>>(base, boxes, cta, rest, nrest, comps, vec, rots, stride);
}

template <int... Cs>
inline void halo_boxes_launch(unsigned grid, cudaStream_t st, double *base, const HaloPatch *boxes, const int2 *cta,
                              const HaloEntry *rest, long long nrest, int comps, int vec, const double *rots,
                              int stride = 0) {
  if (rots && vec != HALO_SCALARS)
    halo_boxes_rot<true, Cs...>(grid, st, base, boxes, cta, rest, nrest, comps, vec, rots, stride);
  else
    halo_boxes_rot<false, Cs...>(grid, st, base, boxes, cta, rest, nrest, comps, vec, rots, stride);
}

__device__ __forceinline__ void unravel(const BlockDev &B, long long t, int &fi, int &fj, int &fk) {
  fi = (int)(t % B.X);
  const long long r = t / B.X;
  fj = (int)(r % B.Y);
  fk = (int)(r / B.Y);
}

// fromQ over the whole block, halo included: the state per cell, the cell's
// last T the starting guess of an iterative eos
// (peregrine/simulator/euler/kernels/state/fromQ.mako:5-19); for the real
// gas its fromrhoE and root Z; with plane set, the double flux's fromplane:
// p off the cell's frozen plane, then the state at rho and p
// (peregrine/simulator/eulerdf/kernels/fromplane.mako:3-17).  With INNER a
// thread a cell of the interior alone (a launch over R_INNER).
template <int NS, bool RG = false, bool INNER = false>
__global__ void k_fromQ(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                        double *__restrict__ stall, const int2 *__restrict__ ctab = nullptr, const int plane = 0) {
  PGB_WHERE(B, u);
  long long t = u;
  if (INNER) {
    if (u >= (long long)B.nx * B.ny * B.nz) return;
    t = cell_index(B, (int)(u % B.nx) + NG, (int)((u / B.nx) % B.ny) + NG, (int)(u / ((long long)B.nx * B.ny)) + NG);
  } else if (t >= B.vol) {
    return;
  }
  const double *Q = Qall + (4 + NS) * B.cv + t;
  double *st = stall + SW * B.cv + t;
  const long long v = B.vol;
  auto Qf = [&](int c) { return Q[c * v]; };
  State s;
  if (RG) {
    const double rho = Qf(0), rhoinv = 1.0 / rho;
    auto Y = [&](int n) { return Qf(5 + n) * rhoinv; };
    const RGMom mom = mixmom_rg<NS>(Y);
    RGState o;
    if (plane) {
      // pplane (peregrine/simulator/mixture/eos/realgasdf/kernels/eos.mako:50-56)
      double composition = 0.0;
#pragma unroll
      for (int n = 0; n < NS - 1; n++) composition += st[(ST_ZETA + n) * v] * Qf(5 + n);
      const double q1 = Qf(1), q2 = Qf(2), q3 = Qf(3);
      const double p = (Qf(4) - 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) * rhoinv - st[ST_EPS * v] * Qf(0) - composition -
                        st[ST_KAPPA * v]) / st[ST_THETA * v];
      o = fromrhop_rg<NS>(mom, Y, rho, p, st[1 * v]);
    } else {
      const double q1 = Qf(1), q2 = Qf(2), q3 = Qf(3);
      const double e = (Qf(4) - 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) * rhoinv) * rhoinv;
      o = fromrhoE_rg<NS>(mom, Y, rho, e, st[1 * v]);
    }
    s = o.s;
    st[ST_Z * v] = o.Z;
  } else {
    s = fromQ<NS>(Qf, st[1 * v]);
  }
  st[0 * v] = s.p, st[1 * v] = s.T, st[2 * v] = s.rhoinv, st[3 * v] = s.rho;
  st[4 * v] = s.e, st[5 * v] = s.cp, st[6 * v] = s.gamma, st[7 * v] = s.c;
}

// the double flux's freeze of one cell (Q and its state record, component
// stride v): the energy reset to the eos's, and the tangent plane of rho e
// at the cell's state, rho e = theta p + eps rho + sum zeta_n rho Y_n + kappa
// (peregrine/simulator/eulerdf/kernels/freeze.mako:3-32)
template <int NS>
__device__ __forceinline__ void freeze_cell(double *Q, double *st, const long long v) {
  const double rho = Q[0], rhoinv = 1.0 / rho;
  const double p = st[0], T = st[1 * v], e = st[4 * v];
  const double rhoe = rho * e;
  Q[4 * v] = rhoe + 0.5 * (Q[1 * v] * Q[1 * v] + Q[2 * v] * Q[2 * v] + Q[3 * v] * Q[3 * v]) * rhoinv;
  auto Y = [&](int n) { return Q[(5 + n) * v] * rhoinv; };
  const RGMom mom = mixmom_rg<NS>(Y);
  double theta, epsY;
  planeslopes<NS>(theta, epsY, mom, Y, rho, rhoinv, T, e);
  double rho_p, rho_T, rho_Y[NS > 1 ? NS - 1 : 1];
  drho_rg<NS>(rho_p, rho_T, rho_Y, mom, Y, p, T, rho);
  double h[NS];
  hspecies_rg<NS>(h, mom, Y, p, T, st[ST_Z * v]);
  const double cpoverrhoT = st[5 * v] / rho_T;
  double zetaY = 0.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double zeta = h[n] - h[NS - 1] - cpoverrhoT * rho_Y[n];
    st[(ST_ZETA + n) * v] = zeta;
    zetaY += zeta * Y(n);
  }
  st[ST_THETA * v] = theta;
  st[ST_EPS * v] = epsY - zetaY;
  st[ST_KAPPA * v] = rhoe - epsY * rho - theta * p;
  (void)rho_p;
}

// the freeze on the interior
template <int NS>
__global__ void k_freeze(const BlockDev *__restrict__ blks, int b, double *__restrict__ Qall,
                         double *__restrict__ stall, const int2 *__restrict__ ctab = nullptr) {
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k);
  freeze_cell<NS>(Qall + (4 + NS) * B.cv + c, stall + SW * B.cv + c, B.vol);
}

__device__ __forceinline__ State load_state(const double *st, long long v) {
  State s;
  s.p = st[0 * v], s.T = st[1 * v], s.rhoinv = st[2 * v], s.rho = st[3 * v];
  s.e = st[4 * v], s.cp = st[5 * v], s.gamma = st[6 * v], s.c = st[7 * v];
  return s;
}

// transport over the whole block: trstate[2 + ns] and hsp[ns] per cell
// (peregrine/simulator/navstokes/kernels/transport.mako:5-35)
template <int NS, bool RG = false>
__global__ void k_transport(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                            const double *__restrict__ stall, double *__restrict__ trall,
                            double *__restrict__ hall, const int2 *__restrict__ ctab = nullptr) {
  PGB_WHERE(B, t);
  if (t >= B.vol) return;
  const double *Q = Qall + (4 + NS) * B.cv + t;
  const State s = load_state(stall + SW * B.cv + t, B.vol);
  double tr[2 + NS], h[NS];
  auto Qf = [&](int c) { return Q[c * B.vol]; };
  transport<NS, decltype(Qf), RG>(Qf, s, tr, h, stall[SW * B.cv + ST_Z * B.vol + t]);
  double *trp = trall + (2 + NS) * B.cv + t;
  double *hp = hall + NS * B.cv + t;
#pragma unroll
  for (int n = 0; n < 2 + NS; n++) trp[n * B.vol] = tr[n];
#pragma unroll
  for (int n = 0; n < NS; n++) hp[n * B.vol] = h[n];
}

// cell gradients of u, v, w, T, Y on the interior
// (peregrine/simulator/navstokes/kernels/dqdxyz.mako:16-41)
// on the interior, or with grow 1 the interior and one halo layer around it
// (the halo's edge cells there read cells no halo fill sets; nothing reads
// their gradients)
template <int NS>
__global__ void k_grads(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                        const double *__restrict__ stall, const double *__restrict__ met,
                        double *__restrict__ gall, int grow = 0,
                        const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS, NGRAD = NE - 1;
  PGB_WHERE(B, t);
  const int gx = B.nx + 2 * grow, gy = B.ny + 2 * grow, gz = B.nz + 2 * grow;
  const long long n = (long long)gx * gy * gz;
  if (t >= n) return;
  const int i = (int)(t % gx) + NG - grow, j = (int)((t / gx) % gy) + NG - grow,
            k = (int)(t / ((long long)gx * gy)) + NG - grow;
  const long long c = cell_index(B, i, j, k);
  const long long sI = 1, sJ = B.X, sK = (long long)B.X * B.Y;
  const double *Q = Qall + NE * B.cv + c;
  const double *T = stall + SW * B.cv + 1 * B.vol + c;
  const double *J = met + M_NCOMP * B.cv + M_JINV * B.vol + c;
  double *g = gall + 3 * NGRAD * B.cv + c;
  const long long v = B.vol;
  const double rIp = Q[sI], rIm = Q[-sI], invI = 1.0 / (rIp * rIm);
  const double rJp = Q[sJ], rJm = Q[-sJ], invJ = 1.0 / (rJp * rJm);
  const double rKp = Q[sK], rKm = Q[-sK], invK = 1.0 / (rKp * rKm);
  double Jm[9];
#pragma unroll
  for (int q = 0; q < 9; q++) Jm[q] = J[q * v];
#pragma unroll
  for (int l = 0; l < NGRAD; l++) {
    double d[3];
    if (l == 3) {
      d[0] = 0.5 * (T[sI] - T[-sI]);
      d[1] = 0.5 * (T[sJ] - T[-sJ]);
      d[2] = 0.5 * (T[sK] - T[-sK]);
    } else {
      const double *Qm = Q + (l + 1) * v;
      d[0] = 0.5 * (Qm[sI] * rIm - Qm[-sI] * rIp) * invI;
      d[1] = 0.5 * (Qm[sJ] * rJm - Qm[-sJ] * rJp) * invJ;
      d[2] = 0.5 * (Qm[sK] * rKm - Qm[-sK] * rKp) * invK;
    }
#pragma unroll
    for (int e = 0; e < 3; e++) g[(3 * l + e) * v] = d[0] * Jm[0 * 3 + e] + d[1] * Jm[1 * 3 + e] + d[2] * Jm[2 * 3 + e];
  }
}

// the interior faces of axis A: face f between cells f - 1 and f
template <int A>
__device__ __forceinline__ bool face_at(const BlockDev &B, long long t, int &i, int &j, int &k) {
  const int fx = B.nx + (A == 0), fy = B.ny + (A == 1), fz = B.nz + (A == 2);
  if (t >= (long long)fx * fy * fz) return false;
  i = (int)(t % fx) + NG;
  j = (int)((t / fx) % fy) + NG;
  k = (int)(t / ((long long)fx * fy)) + NG;
  return true;
}

// the advective face flux, kepaec on the cells as they are
// (peregrine/simulator/euler/kernels/flux/single.mako:4-9 with
//  recon/constant.mako:3-18 and function/kepaec.mako:2-20)
// one face of axis A of a block (Q, st, met the block's own arrays), R the
// index of the cell on its high side, into F[NE]
template <int NS, int A>
__device__ __forceinline__ void advflux_face(const BlockDev &B, const double *__restrict__ Q,
                                             const double *__restrict__ st, const double *__restrict__ met,
                                             const long long R, double *F) {
  const long long L = R - (A == 0 ? 1 : A == 1 ? B.X : (long long)B.X * B.Y);
  const long long v = B.vol;
  const double *S = met + (M_S + 3 * A) * v + R;
  auto side = [&](long long c) {
    const State s = load_state(st + c, v);
    KSide x;
    x.u = Q[1 * v + c] / Q[c];
    x.v = Q[2 * v + c] / Q[c];
    x.w = Q[3 * v + c] / Q[c];
    x.p = s.p, x.rho = s.rho, x.e = s.e;
    x.th = s.cp / s.gamma * s.T;
    return x;
  };
  const KSide sl = side(L), sr = side(R);
  double C;
  kepaec(sl, sr, S[0], S[v], S[2 * v], F, C);
#pragma unroll
  for (int n = 0; n < NS - 1; n++) F[5 + n] = 0.5 * (Q[(5 + n) * v + R] / Q[R] + Q[(5 + n) * v + L] / Q[L]) * C;
}

template <int NS, int A>
__global__ void k_advflux(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                          const double *__restrict__ stall, const double *__restrict__ met,
                          double *__restrict__ Fall, const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS;
  PGB_WHERE(B, t);
  int i, j, k;
  if (!face_at<A>(B, t, i, j, k)) return;
  const long long R = cell_index(B, i, j, k);
  double F[NE];
  advflux_face<NS, A>(B, Qall + NE * B.cv, stall + SW * B.cv, met + M_NCOMP * B.cv, R, F);
  double *Fo = Fall + NE * B.cv + R;
#pragma unroll
  for (int l = 0; l < NE; l++) Fo[l * B.vol] = F[l];
}

// the double flux's kepaec: the plain two-point flux with the energy row
// written twice, in the left cell's frozen plane at F[4] and in the right
// cell's at F[ne] (peregrine/simulator/eulerdf/kernels/flux/function/kepaec.mako:1-21,
// the plain flux function/kepaec.mako:2-20); NE + 1 rows per face
template <int NS, int A>
__device__ __forceinline__ void advflux_df_face(const BlockDev &B, const double *__restrict__ Q,
                                                const double *__restrict__ st, const double *__restrict__ met,
                                                const long long R, double *F) {
  constexpr int NE = 4 + NS;
  const long long L = R - (A == 0 ? 1 : A == 1 ? B.X : (long long)B.X * B.Y);
  const long long v = B.vol;
  const double *Sp = met + (M_S + 3 * A) * v + R;
  const double S0 = Sp[0], S1 = Sp[v], S2 = Sp[2 * v];
  const double uL = Q[1 * v + L] / Q[L], vL = Q[2 * v + L] / Q[L], wL = Q[3 * v + L] / Q[L];
  const double uR = Q[1 * v + R] / Q[R], vR = Q[2 * v + R] / Q[R], wR = Q[3 * v + R] / Q[R];
  const double pL = st[L], pR = st[R], rhoL = st[3 * v + L], rhoR = st[3 * v + R];
  const double uf = 0.5 * (uR + uL), vf = 0.5 * (vR + vL), wf = 0.5 * (wR + wL);
  const double U = S0 * uf + S1 * vf + S2 * wf;
  const double pf = 0.5 * (pR + pL);
  const double rho = 0.5 * (rhoR + rhoL);
  const double C = rho * U;
  F[0] = C;
  F[1] = C * uf + pf * S0;
  F[2] = C * vf + pf * S1;
  F[3] = C * wf + pf * S2;
  const double Kj = C * 0.5 * (uR * uL + vR * vL + wR * wL);
  const double Pj = 0.5 * (pL * (uR * S0 + vR * S1 + wR * S2) + pR * (uL * S0 + vL * S1 + wL * S2));
  double YL[NS > 1 ? NS - 1 : 1], YR[NS > 1 ? NS - 1 : 1];
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    YL[n] = Q[(5 + n) * v + L] / Q[L], YR[n] = Q[(5 + n) * v + R] / Q[R];
    F[5 + n] = 0.5 * (YR[n] + YL[n]) * C;
  }
  const double rhoinvL = 1.0 / rhoL, rhoinvR = 1.0 / rhoR;
  // ecomp: each side's composition energy in each plane
  double cL[2] = {0.0, 0.0}, cR[2] = {0.0, 0.0};
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    const double zL = st[(ST_ZETA + n) * v + L], zR = st[(ST_ZETA + n) * v + R];
    cL[0] += zL * YL[n], cL[1] += zR * YL[n];
    cR[0] += zL * YR[n], cR[1] += zR * YR[n];
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const long long P = q == 0 ? L : R;
    const double theta = st[ST_THETA * v + P], eps = st[ST_EPS * v + P], kappa = st[ST_KAPPA * v + P];
    // ethermal: the thermal part theta p + kappa over the density, at each side's pressure
    const double tL = (theta * pL + kappa) * rhoinvL, tR = (theta * pR + kappa) * rhoinvR;
    F[q == 0 ? 4 : NE] = (eps + 0.5 * (cL[q] + cR[q]) + 2.0 * tL * tR / (tL + tR)) * C + Kj + Pj;
  }
}

template <int NS, int A>
__global__ void k_advflux_df(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                             const double *__restrict__ stall, const double *__restrict__ met,
                             double *__restrict__ Fall, const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS, NF = NE + 1;
  PGB_WHERE(B, t);
  int i, j, k;
  if (!face_at<A>(B, t, i, j, k)) return;
  const long long R = cell_index(B, i, j, k);
  double F[NF];
  advflux_df_face<NS, A>(B, Qall + NE * B.cv, stall + SW * B.cv, met + M_NCOMP * B.cv, R, F);
  double *Fo = Fall + NF * B.cv + R;
#pragma unroll
  for (int l = 0; l < NF; l++) Fo[l * B.vol] = F[l];
}

// the advective face flux of a Riemann solver FN on the cells as they are
// (lim 0; recon/constant.mako:3-18) or on MUSCL's sides under limiter lim
// (recon/muscl.mako:15-51), both sides from the four cells LL, L, R, RR
// along the axis (peregrine/simulator/euler/kernels/flux/single.mako:4-9).
// DF: the double flux's form (Rusanov or AUSM+-up), the energy row written
// again in each of the two cells' frozen planes, F[4] in the left's and
// F[ne] in the right's, from each side's energy in that plane
// (peregrine/simulator/eulerdf/kernels/flux/function/{rusanov,ausmup}.mako,
// eside at peregrine/simulator/mixture/eos/realgasdf/kernels/eos.mako:73-83)
template <int NS, int A, int FN, bool RG = false, bool DF = false>
__device__ __forceinline__ void riemann_face(const BlockDev &B, const double *__restrict__ Q,
                                             const double *__restrict__ st, const double *__restrict__ met,
                                             const int lim, const long long R, double *F) {
  constexpr int NE = 4 + NS, NY = NS > 1 ? NS - 1 : 1;
  const long long d = A == 0 ? 1 : A == 1 ? B.X : (long long)B.X * B.Y;
  const long long L = R - d;
  const long long v = B.vol;
  const double *Sp = met + (M_S + 3 * A) * v + R;
  const double S[3] = {Sp[0], Sp[v], Sp[2 * v]};
  RSide sl, sr;
  double YL[NY], YR[NY];
  if (lim == 0) {
    auto cell = [&](long long c, RSide &x, double *Y) {
      x.p = st[0 * v + c], x.rho = st[3 * v + c], x.e = st[4 * v + c], x.c = st[7 * v + c];
      x.u = Q[1 * v + c] / Q[c];
      x.v = Q[2 * v + c] / Q[c];
      x.w = Q[3 * v + c] / Q[c];
#pragma unroll
      for (int n = 0; n < NS - 1; n++) Y[n] = Q[(5 + n) * v + c] / Q[c];
    };
    cell(L, sl, YL);
    cell(R, sr, YR);
  } else {
    const long long LL = L - d, RR = R + d;
    const double riLL = st[2 * v + LL], riL = st[2 * v + L], riR = st[2 * v + R], riRR = st[2 * v + RR];
    // a row of Q over rho on each side
    auto lft = [&](int row) {
      return muscl_left(lim, Q[row * v + LL] * riLL, Q[row * v + L] * riL, Q[row * v + R] * riR);
    };
    auto rgt = [&](int row) {
      return muscl_right(lim, Q[row * v + L] * riL, Q[row * v + R] * riR, Q[row * v + RR] * riRR);
    };
    // p and T from the state; Y and the velocity as Q times the cell's 1 / rho
    const double pL = muscl_left(lim, st[LL], st[L], st[R]), pR = muscl_right(lim, st[L], st[R], st[RR]);
    const double TL = muscl_left(lim, st[v + LL], st[v + L], st[v + R]);
    const double TR = muscl_right(lim, st[v + L], st[v + R], st[v + RR]);
#pragma unroll
    for (int n = 0; n < NS - 1; n++) YL[n] = lft(5 + n), YR[n] = rgt(5 + n);
    side_frompT<NS, RG>(pL, TL, YL, sl);
    side_frompT<NS, RG>(pR, TR, YR, sr);
    sl.u = lft(1), sl.v = lft(2), sl.w = lft(3);
    sr.u = rgt(1), sr.v = rgt(2), sr.w = rgt(3);
  }
  riemann<FN, NS>(sl, sr, YL, YR, S, F);
  if (DF) {
    // eside: a side's total energy in plane q, theta p + rho (eps + the
    // composition's zeta . Y + |u|^2 / 2) + kappa
    auto eside = [&](const RSide &x, const double *Y, double *E) {
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const long long P = q == 0 ? L : R;
        double comp = 0.0;
#pragma unroll
        for (int n = 0; n < NS - 1; n++) comp += st[(ST_ZETA + n) * v + P] * Y[n];
        E[q] = st[ST_THETA * v + P] * x.p +
               x.rho * (st[ST_EPS * v + P] + comp + 0.5 * (x.u * x.u + x.v * x.v + x.w * x.w)) +
               st[ST_KAPPA * v + P];
      }
    };
    if (FN == FN_RUSANOV) {
      // the plain Rusanov's UL, UR and lam, formed as it forms them
      const double area = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
      const double unL = (sl.u * S[0] + sl.v * S[1] + sl.w * S[2]) / area;
      const double unR = (sr.u * S[0] + sr.v * S[1] + sr.w * S[2]) / area;
      const double lam = fmax(fabs(unL) + sl.c, fabs(unR) + sr.c) * area;
      const double UL = unL * area, UR = unR * area;
      double EpL[2], EpR[2];
      eside(sl, YL, EpL);
      eside(sr, YR, EpR);
#pragma unroll
      for (int q = 0; q < 2; q++)
        F[q == 0 ? 4 : NE] = 0.5 * (UR * (EpR[q] + sr.p) + UL * (EpL[q] + sl.p) - lam * (EpR[q] - EpL[q]));
    } else {
      // AUSM+-up: the mass flux F[0] from the upwind side U
      const double mdot = F[0];
      const bool left = mdot > 0.0;
      const RSide &U = left ? sl : sr;
      const double rhoinvU = 1.0 / U.rho;
      double Ep[2];
      eside(U, left ? YL : YR, Ep);
#pragma unroll
      for (int q = 0; q < 2; q++) F[q == 0 ? 4 : NE] = mdot * (Ep[q] + U.p) * rhoinvU;
    }
  }
}

// F[NE] (NE + 1 rows with DF) of the face of axis A whose high-side cell is R
template <int NS, int A, int FN, bool RG = false, bool DF = false>
__global__ void k_riemann(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                          const double *__restrict__ stall, const double *__restrict__ met,
                          double *__restrict__ Fall, const int lim,
                          const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS, NF = NE + (DF ? 1 : 0);
  PGB_WHERE(B, t);
  int i, j, k;
  if (!face_at<A>(B, t, i, j, k)) return;
  const long long R = cell_index(B, i, j, k);
  double F[NF];
  riemann_face<NS, A, FN, RG, DF>(B, Qall + NE * B.cv, stall + SW * B.cv, met + M_NCOMP * B.cv, lim, R, F);
  double *Fo = Fall + NF * B.cv + R;
#pragma unroll
  for (int l = 0; l < NF; l++) Fo[l * B.vol] = F[l];
}

// the diffusive face flux added to F (peregrine/simulator/navstokes/kernels/flux/alpha-damping.mako:3-99);
// DF: the double flux's faces carry the energy row twice, and the diffusive
// energy flux adds to both (peregrine/simulator/navstokesdf/kernels/flux/alpha-damping.mako:1-9)
// the diffusive rows of the face of axis A whose high-side cell is R added
// to F[NE]; returns the diffusive energy flux (the double flux adds it to its
// second energy row too).  Q, st, tr, hs, gr and M are the block's own arrays.
template <int NS, int A>
__device__ __forceinline__ double diffflux_face(const BlockDev &B, const double *__restrict__ Q,
                                                const double *__restrict__ st, const double *__restrict__ tr,
                                                const double *__restrict__ hs, const double *__restrict__ gr,
                                                const double *__restrict__ M, const long long R, double *F) {
  constexpr int NE = 4 + NS, NGRAD = NE - 1;
  const long long L = R - (A == 0 ? 1 : A == 1 ? B.X : (long long)B.X * B.Y);
  const long long v = B.vol;
  const double S[3] = {M[(M_S + 3 * A) * v + R], M[(M_S + 3 * A + 1) * v + R], M[(M_S + 3 * A + 2) * v + R]};
  const double xf[3] = {M[(M_XF + 3 * A) * v + R], M[(M_XF + 3 * A + 1) * v + R], M[(M_XF + 3 * A + 2) * v + R]};
  const double xL[3] = {M[(M_XCC + 0) * v + L], M[(M_XCC + 1) * v + L], M[(M_XCC + 2) * v + L]};
  const double xR[3] = {M[(M_XCC + 0) * v + R], M[(M_XCC + 1) * v + R], M[(M_XCC + 2) * v + R]};
  const FaceGeom g = face_geom(S[0], S[1], S[2], xf, xL, xR);
  const State sL = load_state(st + L, v), sR = load_state(st + R, v);
  double gL[3 * NGRAD], gRr[3 * NGRAD];
#pragma unroll
  for (int q = 0; q < 3 * NGRAD; q++) gL[q] = gr[q * v + L], gRr[q] = gr[q * v + R];
  const double mu = 0.5 * (tr[0 * v + R] + tr[0 * v + L]);
  const double kappa = 0.5 * (tr[1 * v + R] + tr[1 * v + L]);
  const double lambda = 0.0 - 2.0 / 3.0 * mu;
  const double rhoinvL = sL.rhoinv, rhoinvR = sR.rhoinv;
  const double uL = Q[1 * v + L] * rhoinvL, vL = Q[2 * v + L] * rhoinvL, wL = Q[3 * v + L] * rhoinvL;
  const double uR = Q[1 * v + R] * rhoinvR, vR = Q[2 * v + R] * rhoinvR, wR = Q[3 * v + R] * rhoinvR;
  double dudx, dudy, dudz, dvdx, dvdy, dvdz, dwdx, dwdy, dwdz;
  facegrad(g, uL, uR, gL + 0, gRr + 0, dudx, dudy, dudz);
  facegrad(g, vL, vR, gL + 3, gRr + 3, dvdx, dvdy, dvdz);
  facegrad(g, wL, wR, gL + 6, gRr + 6, dwdx, dwdy, dwdz);
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
  facegrad(g, sL.T, sR.T, gL + 9, gRr + 9, dTx, dTy, dTz);
  const double heatflux = -kappa * (dTx * g.S0 + dTy * g.S1 + dTz * g.S2);
  const double uf = 0.5 * (uR + uL), vf = 0.5 * (vR + vL), wf = 0.5 * (wR + wL);
  double f4 = (uf * txx + vf * txy + wf * txz) * g.S0 + (uf * txy + vf * tyy + wf * tyz) * g.S1 +
              (uf * txz + vf * tyz + wf * tzz) * g.S2 + heatflux;
  double YlastL = 1.0, YlastR = 1.0;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    YlastL -= Q[(5 + n) * v + L] * rhoinvL;
    YlastR -= Q[(5 + n) * v + R] * rhoinvR;
  }
  auto YL = [&](int n) { return n < NS - 1 ? Q[(5 + n) * v + L] * rhoinvL : YlastL; };
  auto YR = [&](int n) { return n < NS - 1 ? Q[(5 + n) * v + R] * rhoinvR : YlastR; };
  double Dk, Vc = 0.0, gradYns = 0.0, sumYh = 0.0, Yns = 1.0;
  const double rho = 0.5 * (Q[R] + Q[L]);
#pragma unroll
  for (int n = 0; n < NS - 1; n++) {
    Dk = 0.5 * (tr[(2 + n) * v + R] + tr[(2 + n) * v + L]);
    double dYx, dYy, dYz;
    facegrad(g, YL(n), YR(n), gL + 3 * (4 + n), gRr + 3 * (4 + n), dYx, dYy, dYz);
    const double gradYk = dYx * g.S0 + dYy * g.S1 + dYz * g.S2;
    gradYns -= gradYk;
    Vc += Dk * gradYk;
    const double Jk = -rho * Dk * gradYk;
    const double hk = 0.5 * (hs[n * v + R] + hs[n * v + L]);
    const double Yk = 0.5 * (YR(n) + YL(n));
    Yns -= Yk;
    sumYh += Yk * hk;
    F[5 + n] += Jk;
    f4 += Jk * hk;
  }
  Dk = 0.5 * (tr[(2 + NS - 1) * v + R] + tr[(2 + NS - 1) * v + L]);
  Vc += Dk * gradYns;
  const double corr = rho * Vc;
#pragma unroll
  for (int n = 0; n < NS - 1; n++) F[5 + n] += 0.5 * (YR(n) + YL(n)) * corr;
  f4 += corr * sumYh;
  const double hns = 0.5 * (hs[(NS - 1) * v + R] + hs[(NS - 1) * v + L]);
  f4 += (-rho * Dk * gradYns + Yns * corr) * hns;
  F[4] += f4;
  return f4;
}

template <int NS, int A, bool DF = false>
__global__ void k_diffflux(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                           const double *__restrict__ stall, const double *__restrict__ trall,
                           const double *__restrict__ hall, const double *__restrict__ gall,
                           const double *__restrict__ met, double *__restrict__ Fall,
                           const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS, NGRAD = NE - 1;
  PGB_WHERE(B, t);
  int i, j, k;
  if (!face_at<A>(B, t, i, j, k)) return;
  const long long R = cell_index(B, i, j, k);
  const long long v = B.vol;
  double F[NE];
  double *Fo = Fall + (NE + (DF ? 1 : 0)) * B.cv + R;
#pragma unroll
  for (int l = 0; l < NE; l++) F[l] = Fo[l * v];
  const double f4 = diffflux_face<NS, A>(B, Qall + NE * B.cv, stall + SW * B.cv, trall + (2 + NS) * B.cv,
                                         hall + NS * B.cv, gall + 3 * NGRAD * B.cv, met + M_NCOMP * B.cv, R, F);
#pragma unroll
  for (int l = 0; l < NE; l++) Fo[l * v] = F[l];
  if (DF) Fo[NE * v] += f4;
}

// dQ = (low faces - high faces) detJinv (peregrine/simulator/advec/kernels/applyflux.mako:2-11)
template <int NS>
__global__ void k_applyflux(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Fi,
                            const double *__restrict__ Fj, const double *__restrict__ Fk,
                            const double *__restrict__ met, double *__restrict__ dQall, int append = 0,
                            const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS;
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k), v = B.vol;
  const long long sJ = B.X, sK = (long long)B.X * B.Y;
  const double detJinv = met[M_NCOMP * B.cv + M_DETJINV * v + c];
  const double *fi = Fi + NE * B.cv + c, *fj = Fj + NE * B.cv + c, *fk = Fk + NE * B.cv + c;
  double *dQ = dQall + NE * B.cv + c;
  // with append, a source began dQ and the fluxes add to it (applyflux.mako's append)
#pragma unroll
  for (int l = 0; l < NE; l++) {
    const double f = (fi[l * v] + fj[l * v] + fk[l * v] - fi[l * v + 1] - fj[l * v + sJ] - fk[l * v + sK]) * detJinv;
    dQ[l * v] = append ? dQ[l * v] + f : f;
  }
}

// the double flux's divergence: the energy row takes F[ne] on the cell's low
// faces, where it is the right cell, and F[4] on its high faces
// (peregrine/simulator/eulerdf/kernels/applyflux.mako:2-14)
template <int NS>
__global__ void k_applyflux_df(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Fi,
                               const double *__restrict__ Fj, const double *__restrict__ Fk,
                               const double *__restrict__ met, double *__restrict__ dQall,
                               const int2 *__restrict__ ctab = nullptr) {
  constexpr int NE = 4 + NS, NF = NE + 1;
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k), v = B.vol;
  const long long sJ = B.X, sK = (long long)B.X * B.Y;
  const double detJinv = met[M_NCOMP * B.cv + M_DETJINV * v + c];
  const double *fi = Fi + NF * B.cv + c, *fj = Fj + NF * B.cv + c, *fk = Fk + NF * B.cv + c;
  double *dQ = dQall + NE * B.cv + c;
#pragma unroll
  for (int l = 0; l < NE; l++) {
    if (l == 4) continue;
    dQ[l * v] = (fi[l * v] + fj[l * v] + fk[l * v] - fi[l * v + 1] - fj[l * v + sJ] - fk[l * v + sK]) * detJinv;
  }
  dQ[4 * v] = (fi[NE * v] + fj[NE * v] + fk[NE * v] - fi[4 * v + 1] - fj[4 * v + sJ] - fk[4 * v + sK]) * detJinv;
}

// one combine (peregrine/integrators/kernels/combine.mako:1-13) on a block's interior
struct CombineDev {
  double *out;
  const double *X[3];
  double w[3];
  double wout;
  int own, nterms, step;
};

static __global__ void k_combine(const BlockDev *__restrict__ blks, int b, int ne, CombineDev cd, const double *__restrict__ dt,
                                 const int2 *__restrict__ ctab = nullptr) {
  PGB_WHERE(B, t);
  if (t >= (long long)B.nx * B.ny * B.nz) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k) + ne * B.cv;
  const double d = *dt;
  for (int l = 0; l < ne; l++) {
    const long long at = c + l * B.vol;
    auto term = [&](int n) { return (cd.step && n == cd.nterms - 1) ? cd.w[n] * d * cd.X[n][at] : cd.w[n] * cd.X[n][at]; };
    double acc;
    int n0;
    if (cd.own) {
      acc = cd.wout * cd.out[at];
      n0 = 0;
    } else {
      acc = term(0);
      n0 = 1;
    }
    for (int n = n0; n < cd.nterms; n++) acc = acc + term(n);
    cd.out[at] = acc;
  }
}

// Q and the state from primitives on the interior (the reference's fromprims);
// the stored T is the next fromQ's starting guess
template <int NS, bool RG = false>
__global__ void k_fromprims(const BlockDev *__restrict__ blks, int b, const double *__restrict__ prims,
                            double *__restrict__ Qall, double *__restrict__ stall) {
  constexpr int NE = 4 + NS;
  const BlockDev &B = blks[b + blockIdx.y];
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)B.nx * B.ny * B.nz;
  if (t >= n) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k);
  double q[NE], Q[NE];
#pragma unroll
  for (int l = 0; l < NE; l++) q[l] = prims[l * n + t];
  State th;
  double Z = 0.0;
  if (RG) {
    const RGState o = frompT_rg<NS>(q[0], q[4], [&](int n) { return q[5 + n]; });
    th = o.s;
    Z = o.Z;
    Q[0] = th.rho;
    Q[1] = th.rho * q[1];
    Q[2] = th.rho * q[2];
    Q[3] = th.rho * q[3];
    Q[4] = th.rho * (th.e + 0.5 * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
#pragma unroll
    for (int n = 0; n < NS - 1; n++) Q[5 + n] = th.rho * q[5 + n];
  } else {
    th = fromprims<NS>(q, Q);
  }
  double *Qo = Qall + NE * B.cv + c;
#pragma unroll
  for (int l = 0; l < NE; l++) Qo[l * B.vol] = Q[l];
  if (stall) {
    double *st = stall + SW * B.cv + c;
    const long long v = B.vol;
    st[0 * v] = th.p, st[1 * v] = th.T, st[2 * v] = th.rhoinv, st[3 * v] = th.rho;
    st[4 * v] = th.e, st[5 * v] = th.cp, st[6 * v] = th.gamma, st[7 * v] = th.c;
    st[ST_Z * v] = Z;
  }
}

// interior cells between a packed host-order buffer [comp][k][j][i] and a register
static __global__ void k_unpack(const BlockDev *__restrict__ blks, int b, int ne, const double *__restrict__ src,
                         double *__restrict__ Rall) {
  const BlockDev &B = blks[b + blockIdx.y];
  const long long n = (long long)B.nx * B.ny * B.nz;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k) + ne * B.cv;
  for (int l = 0; l < ne; l++) Rall[c + l * B.vol] = src[l * n + t];
}

static __global__ void k_pack(const BlockDev *__restrict__ blks, int b, int ne, const double *__restrict__ Rall,
                       double *__restrict__ dst) {
  const BlockDev &B = blks[b + blockIdx.y];
  const long long n = (long long)B.nx * B.ny * B.nz;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k) + ne * B.cv;
  for (int l = 0; l < ne; l++) dst[l * n + t] = Rall[c + l * B.vol];
}

}  // namespace pgb
