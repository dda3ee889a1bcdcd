// The boundary conditions of the per-block path: the halo cells behind every
// block face without a neighbour (the reference's preadvflux hooks), the
// gradients there (postgrads) and the flux through a wall's faces (postflux),
// each a single launch over every boundary face of every block
// (peregrine/simulator/advec/simulator.py:57-84,
//  peregrine/simulator/advecdiff/simulator.py:110-124,
//  peregrine/simulator/euler/kernels/bcs/*.mako,
//  peregrine/simulator/navstokes/kernels/bcs/*.mako).
//
// A boundary pass's threads run over its faces end to end; a face's threads
// over its halo layers (layer 0 next to the face) and, inside a layer, over
// the face's cells with the in-plane axis of the smaller stride fastest.  The
// cells a thread reads follow the reference's carried offsets
// (peregrine/launch/policy.py:143-232): "interior" is the first cell in from
// the face whatever the layer, "mirror" the layer's image through the face
// (layer l reads depth l, clamped to the block's deepest cell), "mirror1" one
// deeper, and "intface" the boundary face itself.  Edges and corners of the
// halo are not boundary cells (peregrine/launch/ranges.py:32-40).
#pragma once
#include "bc_types.h"
#include "layout.cuh"
#include "physics.cuh"
#include "plain.cuh"

namespace pgb {

// a value's program at the face centre x and time t: the reference renders its
// expressions of x, y, z and t as C++ (peregrine/simulator/bcs.py:101-143);
// here the same expression runs on a stack.  The host checked every program's
// depth; a malformed one still stays inside the stack and gives NaN.
__device__ inline double bc_eval(const BcOp *__restrict__ ops, const int first, const int end, const double *x,
                                 const double t) {
  double st[PGB_BC_STACK];
  int sp = 0;
  for (int k = first; k < end; k++) {
    const int op = ops[k].op;
    if (op <= PGB_OP_T) {
      if (sp >= PGB_BC_STACK) return nan("");
      st[sp++] = op == PGB_OP_CONST ? ops[k].arg : op == PGB_OP_T ? t : x[op - PGB_OP_X];
      continue;
    }
    const bool binary = op == PGB_OP_ADD || op == PGB_OP_SUB || op == PGB_OP_MUL || op == PGB_OP_DIV ||
                        op == PGB_OP_POW || op == PGB_OP_MIN || op == PGB_OP_MAX;
    if (sp < (binary ? 2 : 1)) return nan("");
    if (binary) {
      const double b = st[--sp], a = st[sp - 1];
      double r;
      switch (op) {
        case PGB_OP_ADD: r = a + b; break;
        case PGB_OP_SUB: r = a - b; break;
        case PGB_OP_MUL: r = a * b; break;
        case PGB_OP_DIV: r = a / b; break;
        case PGB_OP_POW: r = pow(a, b); break;
        case PGB_OP_MIN: r = fmin(a, b); break;
        default: r = fmax(a, b); break;
      }
      st[sp - 1] = r;
      continue;
    }
    const double a = st[sp - 1];
    double r;
    switch (op) {
      case PGB_OP_NEG: r = -a; break;
      case PGB_OP_SIN: r = sin(a); break;
      case PGB_OP_COS: r = cos(a); break;
      case PGB_OP_TAN: r = tan(a); break;
      case PGB_OP_EXP: r = exp(a); break;
      case PGB_OP_LOG: r = log(a); break;
      case PGB_OP_SQRT: r = sqrt(a); break;
      case PGB_OP_TANH: r = tanh(a); break;
      case PGB_OP_ABS: r = fabs(a); break;
      default: return nan("");
    }
    st[sp - 1] = r;
  }
  return sp == 1 ? st[0] : nan("");
}

// the face of a pass thread t works on: faces[f].start <= t < faces[f + 1].start
__device__ inline int bc_face_of(const BcFace *__restrict__ faces, const int nfaces, const long long t) {
  int lo = 0, hi = nfaces;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (faces[mid].start <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// where a boundary thread's cells lie along the face's axis a: the index of
// the cell d deep from the face, the halo cell of layer l, and the face
struct BcAt {
  int a, low;
  int n[3];
  int ij[3];  // the in-plane indices (the axis a entry is set per use)
  __device__ long long cell(const BlockDev &B, int along) const {
    int c[3] = {ij[0], ij[1], ij[2]};
    c[a] = along;
    return cell_index(B, c[0], c[1], c[2]);
  }
  __device__ long long deep(const BlockDev &B, int d) const {
    d = min(d, n[a] - 1);
    return cell(B, low ? NG + d : NG + n[a] - 1 - d);
  }
  __device__ long long halo(const BlockDev &B, int layer) const {
    return cell(B, low ? NG - 1 - layer : NG + n[a] + layer);
  }
  // the face array's index of the boundary face (a face indexed like the cell to its right)
  __device__ long long face(const BlockDev &B) const { return cell(B, low ? NG : NG + n[a]); }
};

// thread q of a face's layer: the face's cell (q1, q2), the in-plane axis of
// the smaller stride fastest
__device__ inline BcAt bc_at(const BlockDev &B, const int face, const long long q) {
  BcAt w;
  w.a = face >> 1;
  w.low = (face & 1) == 0;
  w.n[0] = B.nx, w.n[1] = B.ny, w.n[2] = B.nz;
  const int a1 = w.a == 0 ? 1 : 0, a2 = w.a == 2 ? 1 : 2;
  w.ij[a1] = NG + (int)(q % w.n[a1]);
  w.ij[a2] = NG + (int)(q / w.n[a1]);
  w.ij[w.a] = 0;
  return w;
}

__device__ inline long long bc_plane(const BlockDev &B, const int face) {
  const int a = face >> 1;
  const int n[3] = {B.nx, B.ny, B.nz};
  return (long long)n[a == 0 ? 1 : 0] * n[a == 2 ? 1 : 2];
}

// a cell's Q and state, components vol apart
template <int NE>
__device__ inline void bc_loadQ(const double *Qb, long long c, long long v, double *Q) {
#pragma unroll
  for (int l = 0; l < NE; l++) Q[l] = Qb[l * v + c];
}

// fromprims into a halo cell (peregrine/simulator/euler/kernels/solution.mako:14-23):
// the eos's state at p and T, Q from it and the velocity, the carried species
// from the mass fractions Y (n < ns - 1)
template <int NS, bool RG, class YF>
__device__ inline void bc_fromprims(const double p, const double T, const double *u, YF Y, double *Q, State &th,
                                    double &Z) {
  if (RG) {
    const RGState o = frompT_rg<NS>(p, T, Y);
    th = o.s, Z = o.Z;
  } else {
    th = frompT<NS>(p, T, Y), Z = 0.0;
  }
  Q[0] = th.rho;
  Q[1] = th.rho * u[0];
  Q[2] = th.rho * u[1];
  Q[3] = th.rho * u[2];
  Q[4] = th.rho * (th.e + 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
#pragma unroll
  for (int n = 0; n < NS - 1; n++) Q[5 + n] = th.rho * Y(n);
}

// the outward (sign 1) or inward (sign -1) unit normal of a boundary face,
// sign = outward for the outward one
__device__ inline void bc_normal(const double *S, const double sign, double *nrm) {
  const double Sinv = sign / sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
  nrm[0] = S[0] * Sinv, nrm[1] = S[1] * Sinv, nrm[2] = S[2] * Sinv;
}

// the outflows' halo velocity: extrapolated from the first cell where its
// flow leaves, the mirror's image through the face where it comes back in
// (peregrine/simulator/euler/kernels/bcs/sub-out-fp.mako:17-30)
__device__ inline void bc_outvelocity(const double *Qi, const double rhoinv, const double *Qm, const double *Qm1,
                                      const double *nrm, double *u) {
  const double u0[3] = {Qi[1] * rhoinv, Qi[2] * rhoinv, Qi[3] * rhoinv};
  const double un = u0[0] * nrm[0] + u0[1] * nrm[1] + u0[2] * nrm[2];
  if (un > 0.0) {
    const double rhoinv1 = 1.0 / Qm1[0];
#pragma unroll
    for (int d = 0; d < 3; d++) u[d] = 2.0 * u0[d] - Qm1[1 + d] * rhoinv1;
  } else {
    const double rhoinvm = 1.0 / Qm[0];
    const double um[3] = {Qm[1] * rhoinvm, Qm[2] * rhoinvm, Qm[3] * rhoinvm};
    const double umn = 2.0 * (um[0] * nrm[0] + um[1] * nrm[1] + um[2] * nrm[2]);
    u[0] = um[0] - umn * nrm[0];
    u[1] = um[1] - umn * nrm[1];
    u[2] = um[2] - umn * nrm[2];
  }
}

// preadvflux: every halo cell behind every boundary face, Q and the state
// (the kinds' preadvflux kernels, peregrine/simulator/euler/kernels/bcs/*.mako
// and the Navier-Stokes walls' stuckhalo and stuckhaloisot,
// peregrine/simulator/navstokes/kernels/bcs/wall.mako:7-38)
template <int NS, bool RG>
__global__ void k_bc_halo(const BlockDev *__restrict__ blks, const BcFace *__restrict__ faces, int nfaces,
                          const BcEntry *__restrict__ entries, const BcOp *__restrict__ ops,
                          double *__restrict__ Qall, double *__restrict__ stall, const double *__restrict__ met,
                          const double *__restrict__ clock, const double *__restrict__ dt, double tfrac) {
  constexpr int NE = 4 + NS;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= faces[nfaces].start) return;
  const int f = bc_face_of(faces, nfaces, t);
  const BcFace F = faces[f];
  const BlockDev &B = blks[F.blk];
  const BcEntry &E = entries[F.entry];
  const long long plane = bc_plane(B, F.face), local = t - F.start;
  const int layer = (int)(local / plane);
  const BcAt w = bc_at(B, F.face, local % plane);
  const long long v = B.vol;
  const double *Qb = Qall + NE * B.cv;
  const double *sb = stall + SW * B.cv;
  const double *mb = met + M_NCOMP * B.cv;
  const long long fc = w.face(B);
  const double S[3] = {mb[(M_S + 3 * w.a + 0) * v + fc], mb[(M_S + 3 * w.a + 1) * v + fc],
                       mb[(M_S + 3 * w.a + 2) * v + fc]};
  const double xf[3] = {mb[(M_XF + 3 * w.a + 0) * v + fc], mb[(M_XF + 3 * w.a + 1) * v + fc],
                        mb[(M_XF + 3 * w.a + 2) * v + fc]};
  const double outward = w.low ? -1.0 : 1.0;
  const double tme = *clock + tfrac * *dt;
  double val[BC_MAXV];
  for (int k = 0; k < E.nval; k++) val[k] = bc_eval(ops, E.start[k], E.start[k + 1], xf, tme);
  const long long ci = w.deep(B, 0), cm = w.deep(B, layer), cm1 = w.deep(B, layer + 1);
  double Qi[NE], Qm[NE], Qh[NE];
  bc_loadQ<NE>(Qb, ci, v, Qi);
  bc_loadQ<NE>(Qb, cm, v, Qm);
  State th;
  double Z = 0.0;
  bool copy = false;  // the halo's state is the mirror's as stored
  const int kind = E.kind;
  if (kind == PGB_BC_SLIP_ADIA_WALL) {
    // the momentum's normal part taken off twice; energy and state the image's
    // (peregrine/simulator/euler/kernels/bcs/slp-adia-wall.mako:4-22)
    double nrm[3];
    bc_normal(S, 1.0, nrm);
    const double mn = 2.0 * (Qm[1] * nrm[0] + Qm[2] * nrm[1] + Qm[3] * nrm[2]);
    Qh[0] = Qm[0];
    Qh[1] = Qm[1] - mn * nrm[0];
    Qh[2] = Qm[2] - mn * nrm[1];
    Qh[3] = Qm[3] - mn * nrm[2];
    Qh[4] = Qm[4];
#pragma unroll
    for (int n = 0; n < NS - 1; n++) Qh[5 + n] = Qm[5 + n];
    copy = true;
  } else if (kind == PGB_BC_NOSLIP_ADIA_WALL || kind == PGB_BC_MOV_ADIA_WALL) {
    // stuckhalo: the velocity 2 wall - u at the image's density, the energy
    // moved by the kinetic energy's change, the state the image's
    const double wall[3] = {kind == PGB_BC_MOV_ADIA_WALL ? val[0] : 0.0, kind == PGB_BC_MOV_ADIA_WALL ? val[1] : 0.0,
                            kind == PGB_BC_MOV_ADIA_WALL ? val[2] : 0.0};
    const double rho = Qm[0], rhoinv = 1.0 / rho;
    double ke = 0.0, kehalo = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double u = Qm[1 + d] * rhoinv, uh = 2.0 * wall[d] - u;
      Qh[1 + d] = rho * uh;
      ke += u * u;
      kehalo += uh * uh;
    }
    Qh[0] = rho;
    Qh[4] = Qm[4] + 0.5 * rho * (kehalo - ke);
#pragma unroll
    for (int n = 0; n < NS - 1; n++) Qh[5 + n] = Qm[5 + n];
    copy = true;
  } else if (kind == PGB_BC_SUB_IN_FMT) {
    // the halo velocity makes the face's averages of density and velocity
    // carry the entry's mass flux (sub-in-fmt.mako:4-30)
    double nrm[3];
    bc_normal(S, -outward, nrm);
    const double p = 2.0 * sb[ci] - sb[cm1], T = val[1];
    auto Y = [&](int n) { return val[2 + n]; };
    if (RG) {
      const RGState o = frompT_rg<NS>(p, T, Y);
      th = o.s, Z = o.Z;
    } else {
      th = frompT<NS>(p, T, Y);
    }
    const double rhoinv = 1.0 / Qi[0];
    const double scale = 4.0 * val[0] / (Qi[0] + th.rho);
    const double u[3] = {nrm[0] * scale - Qi[1] * rhoinv, nrm[1] * scale - Qi[2] * rhoinv,
                         nrm[2] * scale - Qi[3] * rhoinv};
    Qh[0] = th.rho;
    Qh[1] = th.rho * u[0];
    Qh[2] = th.rho * u[1];
    Qh[3] = th.rho * u[2];
    Qh[4] = th.rho * (th.e + 0.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
#pragma unroll
    for (int n = 0; n < NS - 1; n++) Qh[5 + n] = th.rho * Y(n);
  } else {
    // the kinds that set the halo by fromprims at a pressure, temperature,
    // velocity and composition
    double p, T, u[3];
    double Yv[NS > 1 ? NS - 1 : 1];
    if (kind == PGB_BC_SLIP_ISOT_WALL) {
      // the velocity mirrored, the image's pressure and composition at the
      // wall's temperature (slp-isot-wall.mako:5-20)
      double nrm[3];
      bc_normal(S, 1.0, nrm);
      const double rhoinv = 1.0 / Qm[0];
      const double ui = Qm[1] * rhoinv, vi = Qm[2] * rhoinv, wi = Qm[3] * rhoinv;
      const double un = 2.0 * (ui * nrm[0] + vi * nrm[1] + wi * nrm[2]);
      u[0] = ui - un * nrm[0], u[1] = vi - un * nrm[1], u[2] = wi - un * nrm[2];
      p = sb[cm], T = val[0];
#pragma unroll
      for (int n = 0; n < NS - 1; n++) Yv[n] = Qm[5 + n] * rhoinv;
    } else if (kind == PGB_BC_NOSLIP_ISOT_WALL || kind == PGB_BC_MOV_ISOT_WALL) {
      // stuckhaloisot (navstokes/kernels/bcs/wall.mako:27-38)
      const bool mov = kind == PGB_BC_MOV_ISOT_WALL;
      const double rhoinv = 1.0 / Qm[0];
#pragma unroll
      for (int d = 0; d < 3; d++) u[d] = 2.0 * (mov ? val[d] : 0.0) - Qm[1 + d] * rhoinv;
      p = sb[cm], T = mov ? val[3] : val[0];
#pragma unroll
      for (int n = 0; n < NS - 1; n++) Yv[n] = Qm[5 + n] * rhoinv;
    } else if (kind == PGB_BC_SUB_IN_FVT) {
      // the pressure extrapolated, the rest the entry's (sub-in-fvt.mako:4-14)
      p = 2.0 * sb[ci] - sb[cm1], T = val[3];
      u[0] = val[0], u[1] = val[1], u[2] = val[2];
#pragma unroll
      for (int n = 0; n < NS - 1; n++) Yv[n] = val[4 + n];
    } else if (kind == PGB_BC_SUP_IN_FA) {
      // everything the entry's (sup-in-fa.mako:4-13)
      p = val[0], T = val[4];
      u[0] = val[1], u[1] = val[2], u[2] = val[3];
#pragma unroll
      for (int n = 0; n < NS - 1; n++) Yv[n] = val[5 + n];
    } else if (kind == PGB_BC_SUB_IN_FTPTT) {
      // total pressure and temperature: the outgoing invariant on the first
      // cell's gamma and c, the total enthalpy by the eos
      // (sub-in-ftptt.mako:4-45)
      double nrm[3];
      bc_normal(S, -outward, nrm);
      const State si = load_state(sb + ci, v);
      const double gamma = si.gamma, c = si.c, gm1 = gamma - 1.0;
      const double rhoinv = 1.0 / Qi[0];
      const double u0[3] = {Qi[1] * rhoinv, Qi[2] * rhoinv, Qi[3] * rhoinv};
      auto Yin = [&](int n) { return val[2 + n]; };
      const double Ttotal = val[1];
      const State total = frompT<NS, decltype(Yin), RG>(si.p, Ttotal, Yin);
      const State cell = frompT<NS, decltype(Yin), RG>(si.p, si.T, Yin);
      const double Ht = c * c / gm1 + (total.e + total.p / total.rho) - (cell.e + cell.p / cell.rho);
      const double Un = u0[0] * nrm[0] + u0[1] * nrm[1] + u0[2] * nrm[2];
      const double Jm = -Un + 2.0 * c / gm1;
      const double aq = 1.0 + 2.0 / gm1;
      const double bq = -2.0 * Jm;
      const double cq = gm1 * (0.5 * Jm * Jm - Ht);
      const double t1 = -bq / (2.0 * aq);
      const double t2 = sqrt(fmax(bq * bq - 4.0 * aq * cq, 0.0)) / (2.0 * aq);
      const double cb = fmax(t1 + t2, t1 - t2);
      const double Vb = 2.0 * cb / gm1 - Jm;
      const double Mb = Vb / cb;
      const double isentropic = 1.0 + 0.5 * gm1 * Mb * Mb;
      p = val[0] * pow(isentropic, -gamma / gm1), T = Ttotal / isentropic;
      u[0] = Vb * nrm[0], u[1] = Vb * nrm[1], u[2] = Vb * nrm[2];
#pragma unroll
      for (int n = 0; n < NS - 1; n++) Yv[n] = val[2 + n];
    } else {
      // the outflows (sub-out-fp.mako:4-41, sup-out-fn.mako:4-48)
      double nrm[3];
      bc_normal(S, outward, nrm);
      double Qm1[NE];
      bc_loadQ<NE>(Qb, cm1, v, Qm1);
      const double rhoinv = 1.0 / Qi[0];
      bc_outvelocity(Qi, rhoinv, Qm, Qm1, nrm, u);
      if (kind == PGB_BC_SUB_OUT_FP) {
        p = val[0], T = sb[v + ci];
#pragma unroll
        for (int n = 0; n < NS - 1; n++) Yv[n] = Qi[5 + n] * rhoinv;
      } else {
        // the pressure capped at the interior's so a wave can only leave; the
        // floors a hundredth of the interior's
        const double rhoinv1 = 1.0 / Qm1[0];
        const double least = 0.01;
        const double p0 = sb[ci], T0 = sb[v + ci];
        p = fmin(fmax(least * p0, 2.0 * p0 - sb[cm1]), p0);
        T = fmax(least * T0, 2.0 * T0 - sb[v + cm1]);
#pragma unroll
        for (int n = 0; n < NS - 1; n++) Yv[n] = fmax(0.0, fmin(1.0, 2.0 * Qi[5 + n] * rhoinv - Qm1[5 + n] * rhoinv1));
      }
    }
    auto Y = [&](int n) { return Yv[n]; };
    bc_fromprims<NS, RG>(p, T, u, Y, Qh, th, Z);
  }
  const long long ch = w.halo(B, layer);
  double *Qo = Qall + NE * B.cv + ch;
#pragma unroll
  for (int l = 0; l < NE; l++) Qo[l * v] = Qh[l];
  double *so = stall + SW * B.cv + ch;
  if (copy) {
    const double *sm = sb + cm;
#pragma unroll
    // the whole record, the double flux's plane with it (the reference's
    // statehalo.copy, every field of the state array)
#pragma unroll
    for (int q = 0; q < ST_ZETA + NS - 1; q++) so[q * v] = sm[q * v];
  } else {
    so[0 * v] = th.p, so[1 * v] = th.T, so[2 * v] = th.rhoinv, so[3 * v] = th.rho;
    so[4 * v] = th.e, so[5 * v] = th.cp, so[6 * v] = th.gamma, so[7 * v] = th.c;
    so[ST_Z * v] = Z;
  }
}

// the double flux's freeze of the boundaries' halo cells, once the halo pass
// has set them at a step's start: a halo cell carries the plane of its own
// state, as the reference's freeze over every cell gives it
// (peregrine/simulator/eulerdf/simulator.py:58-66)
template <int NS>
__global__ void k_bc_freeze(const BlockDev *__restrict__ blks, const BcFace *__restrict__ faces, int nfaces,
                            double *__restrict__ Qall, double *__restrict__ stall) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= faces[nfaces].start) return;
  const int f = bc_face_of(faces, nfaces, t);
  const BcFace F = faces[f];
  const BlockDev &B = blks[F.blk];
  const long long plane = bc_plane(B, F.face), local = t - F.start;
  const int layer = (int)(local / plane);
  const BcAt w = bc_at(B, F.face, local % plane);
  const long long ch = w.halo(B, layer);
  freeze_cell<NS>(Qall + (4 + NS) * B.cv + ch, stall + SW * B.cv + ch, B.vol);
}

// postgrads of the inflows and outflows: each halo cell's gradients its
// image's (peregrine/simulator/navstokes/kernels/bcs/gradients.mako:2-6)
template <int NS>
__global__ void k_bc_grads(const BlockDev *__restrict__ blks, const BcFace *__restrict__ faces, int nfaces,
                           double *__restrict__ gall) {
  constexpr int NG3 = 3 * (3 + NS);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= faces[nfaces].start) return;
  const int f = bc_face_of(faces, nfaces, t);
  const BcFace F = faces[f];
  const BlockDev &B = blks[F.blk];
  const long long plane = bc_plane(B, F.face), local = t - F.start;
  const int layer = (int)(local / plane);
  const BcAt w = bc_at(B, F.face, local % plane);
  const long long v = B.vol;
  double *g = gall + NG3 * B.cv;
  const long long cm = w.deep(B, layer), ch = w.halo(B, layer);
#pragma unroll
  for (int q = 0; q < NG3; q++) g[q * v + ch] = g[q * v + cm];
}

// postflux of the walls: the flux through each wall face written from the
// first cell in, over the flux function's: the acoustic wall pressure
// (peregrine/simulator/euler/kernels/bcs/wall.mako:2-16) and, with viscosity,
// the wall's shear stress from the normal derivative of the velocity, its
// work and, on an isothermal wall, the heat flux at the wall's temperature
// (peregrine/simulator/navstokes/kernels/bcs/wall.mako:40-99)
template <int NS>
__global__ void k_bc_wall(const BlockDev *__restrict__ blks, const BcFace *__restrict__ faces, int nfaces,
                          const BcEntry *__restrict__ entries, const BcOp *__restrict__ ops,
                          const double *__restrict__ Qall, const double *__restrict__ stall,
                          const double *__restrict__ trall, const double *__restrict__ met, double *Fi, double *Fj,
                          double *Fk, int nf, int visc, const double *__restrict__ clock,
                          const double *__restrict__ dt, double tfrac) {
  constexpr int NE = 4 + NS;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= faces[nfaces].start) return;
  const int f = bc_face_of(faces, nfaces, t);
  const BcFace Fc = faces[f];
  const BlockDev &B = blks[Fc.blk];
  const BcEntry &E = entries[Fc.entry];
  const BcAt w = bc_at(B, Fc.face, t - Fc.start);
  const long long v = B.vol;
  const double *mb = met + M_NCOMP * B.cv;
  const long long fc = w.face(B), ci = w.deep(B, 0);
  const double S[3] = {mb[(M_S + 3 * w.a + 0) * v + fc], mb[(M_S + 3 * w.a + 1) * v + fc],
                       mb[(M_S + 3 * w.a + 2) * v + fc]};
  const double xf[3] = {mb[(M_XF + 3 * w.a + 0) * v + fc], mb[(M_XF + 3 * w.a + 1) * v + fc],
                        mb[(M_XF + 3 * w.a + 2) * v + fc]};
  const double outward = w.low ? -1.0 : 1.0;
  double Q[NE];
  bc_loadQ<NE>(Qall + NE * B.cv, ci, v, Q);
  const State st = load_state(stall + SW * B.cv + ci, v);
  double Fo[NE + 1];
  // wallpressure: p + rho c u_n, a Riemann solver's star pressure to first order
  const double area = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
  const double un = outward * (Q[1] * S[0] + Q[2] * S[1] + Q[3] * S[2]) / (Q[0] * area);
  const double pw = fmax(st.p + Q[0] * st.c * un, 0.0);
  Fo[0] = 0.0;
  Fo[1] = pw * S[0];
  Fo[2] = pw * S[1];
  Fo[3] = pw * S[2];
  for (int l = 4; l < nf; l++) Fo[l] = 0.0;
  if (visc) {
    const int kind = E.kind;
    const double tme = *clock + tfrac * *dt;
    double val[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < E.nval && k < 4; k++) val[k] = bc_eval(ops, E.start[k], E.start[k + 1], xf, tme);
    const bool mov = kind == PGB_BC_MOV_ADIA_WALL || kind == PGB_BC_MOV_ISOT_WALL;
    const bool isot = kind == PGB_BC_SLIP_ISOT_WALL || kind == PGB_BC_NOSLIP_ISOT_WALL || kind == PGB_BC_MOV_ISOT_WALL;
    const double stuck = (kind == PGB_BC_SLIP_ADIA_WALL || kind == PGB_BC_SLIP_ISOT_WALL) ? 0.0 : 1.0;
    const double wall[3] = {mov ? val[0] : 0.0, mov ? val[1] : 0.0, mov ? val[2] : 0.0};
    double mu, kappa, dT;
    if (isot) {
      // wallcoeffs: mu and kappa of the first cell's composition at the wall's
      // temperature and the first cell's pressure
      const double Tw = kind == PGB_BC_MOV_ISOT_WALL ? val[3] : val[0];
      const double rhoinv = 1.0 / Q[0];
      auto Yc = [&](int n) { return Q[5 + n] * rhoinv; };
      const State at = frompT<NS>(st.p, Tw, Yc);
      auto Qf = [&](int c) { return Q[c]; };
      double tr[2 + NS], h[NS];
      transport<NS>(Qf, at, tr, h);
      mu = tr[0], kappa = tr[1], dT = Tw - st.T;
    } else {
      const double *tr = trall + (2 + NS) * B.cv + ci;
      mu = tr[0], kappa = tr[v], dT = 0.0;
    }
    const double xc[3] = {mb[(M_XCC + 0) * v + ci], mb[(M_XCC + 1) * v + ci], mb[(M_XCC + 2) * v + ci]};
    const double Sabs = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]), Sinv = 1.0 / Sabs;
    const double n[3] = {S[0] * Sinv, S[1] * Sinv, S[2] * Sinv};
    const double dn = fabs((xc[0] - xf[0]) * n[0] + (xc[1] - xf[1]) * n[1] + (xc[2] - xf[2]) * n[2]);
    const double rhoinv = 1.0 / Q[0];
    double dun[3];
#pragma unroll
    for (int d = 0; d < 3; d++) dun[d] = outward * (wall[d] - Q[1 + d] * rhoinv) / dn;
    const double div = dun[0] * n[0] + dun[1] * n[1] + dun[2] * n[2];
    // every component where the flow is held, the normal one alone where it slips
#pragma unroll
    for (int d = 0; d < 3; d++) dun[d] = div * n[d] + stuck * (dun[d] - div * n[d]);
    double work = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double tS = -mu * Sabs * (dun[d] + div * n[d] / 3.0);
      Fo[1 + d] += tS;
      work += wall[d] * tS;
    }
    Fo[4] += work - kappa * outward * dT / dn * Sabs;
  }
  // the double flux's second energy row: nothing is advected through a wall,
  // so it is the first's (peregrine/simulator/navstokesdf/kernels/bcs/*-wall.mako)
  if (nf > NE) Fo[NE] = Fo[4];
  double *Fa = (w.a == 0 ? Fi : w.a == 1 ? Fj : Fk) + (long long)nf * B.cv + fc;
  for (int l = 0; l < nf; l++) Fa[l * v] = Fo[l];
}

}  // namespace pgb
