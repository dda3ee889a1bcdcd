// The CFL reduction: the largest acoustic, convective and combined CFL number
// per unit step over every block's interior (the reference's cflmax kernel,
// peregrine/simulator/euler/kernels/cflmax.mako:2-33, with the cell lengths of
// peregrine/multiblock/block/grid.py:164-176), and the cfl controller's step
// size from it (peregrine/integrators/controllers.py:21-30), both on the
// device so a stepping loop under the controller needs no host round trip.
#pragma once
#include "layout.cuh"
#include "physics.cuh"
#include "plain.cuh"

namespace pgb {

// a non-negative double's bit pattern orders as an unsigned integer does
__device__ inline void cfl_atomic_max(double *slot, const double v) {
  atomicMax(reinterpret_cast<unsigned long long *>(slot), (unsigned long long)__double_as_longlong(v));
}

// one thread per interior cell of each block; the sound speed of the state
// fromQ makes of Q (the cell's stored T as the iterative eos's starting
// guess when there is a state; with plane, the double flux's p off the
// cell's frozen plane); each CTA's maxima folded into out[0..2] (acoustic,
// convective, combined), which the caller zeroed.  A NaN cell is passed
// over, as fmax passes it.
template <int NS, bool RG>
__device__ inline void cfl_cell(const BlockDev &B, const long long t, const double *__restrict__ Qall,
                                const double *__restrict__ stall, const double *__restrict__ met, const int plane,
                                double *m) {
  constexpr int NE = 4 + NS;
  const int i = (int)(t % B.nx) + NG, j = (int)((t / B.nx) % B.ny) + NG, k = (int)(t / ((long long)B.nx * B.ny)) + NG;
  const long long c = cell_index(B, i, j, k), v = B.vol;
  const double *Q = Qall + NE * B.cv + c;
  auto Qf = [&](int l) { return Q[l * v]; };
  const double *st = stall ? stall + SW * B.cv + c : nullptr;
  const double Tg = st ? st[1 * v] : 0.0;
  double cs;
  if (RG) {
    const double rho = Qf(0), rhoinv = 1.0 / rho;
    auto Y = [&](int n) { return Qf(5 + n) * rhoinv; };
    const RGMom mom = mixmom_rg<NS>(Y);
    const double q1 = Qf(1), q2 = Qf(2), q3 = Qf(3);
    if (plane && st) {
      double composition = 0.0;
#pragma unroll
      for (int n = 0; n < NS - 1; n++) composition += st[(ST_ZETA + n) * v] * Qf(5 + n);
      const double p = (Qf(4) - 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) * rhoinv - st[ST_EPS * v] * Qf(0) -
                        composition - st[ST_KAPPA * v]) / st[ST_THETA * v];
      cs = fromrhop_rg<NS>(mom, Y, rho, p, Tg).s.c;
    } else {
      const double e = (Qf(4) - 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) * rhoinv) * rhoinv;
      cs = fromrhoE_rg<NS>(mom, Y, rho, e, Tg).s.c;
    }
  } else {
    cs = fromQ<NS>(Qf, Tg).c;
  }
  const int n[3] = {B.nx, B.ny, B.nz};
  const double rhoinv = 1.0 / Qf(0);
  const double vel[3] = {Qf(1) * rhoinv, Qf(2) * rhoinv, Qf(3) * rhoinv};
  double d[3], un[3];
  if (B.uniform) {
    // a uniform block's faces are its axes and its cells one length per
    // axis: the unit normals' mean is the axis, the length the spacing
#pragma unroll
    for (int a = 0; a < 3; a++) {
      d[a] = n[a] == 1 ? (double)INFINITY : fabs(B.ex[a]);
      un[a] = fabs(vel[a]);
    }
  } else {
    const double *mb = met + M_NCOMP * B.cv;
    const long long step[3] = {1, B.X, (long long)B.X * B.Y};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double *S = mb + (M_S + 3 * a) * v + c;
      const double *xf = mb + (M_XF + 3 * a) * v + c;
      const long long h = step[a];
      // the length between the cell's two face centres; an axis one cell
      // thick is not marched in: infinitely long, so it limits nothing
      const double s0 = xf[0 * v + h] - xf[0 * v], s1 = xf[1 * v + h] - xf[1 * v], s2 = xf[2 * v + h] - xf[2 * v];
      d[a] = n[a] == 1 ? (double)INFINITY : sqrt(s0 * s0 + s1 * s1 + s2 * s2);
      // the normal velocity on the mean of the two faces' unit normals
      const double L0 = S[0 * v], L1 = S[1 * v], L2 = S[2 * v];
      const double H0 = S[0 * v + h], H1 = S[1 * v + h], H2 = S[2 * v + h];
      const double S0inv = 1.0 / sqrt(L0 * L0 + L1 * L1 + L2 * L2);
      const double S1inv = 1.0 / sqrt(H0 * H0 + H1 * H1 + H2 * H2);
      const double nx = 0.5 * (L0 * S0inv + H0 * S1inv);
      const double ny = 0.5 * (L1 * S0inv + H1 * S1inv);
      const double nz = 0.5 * (L2 * S0inv + H2 * S1inv);
      un[a] = fabs(nx * vel[0] + ny * vel[1] + nz * vel[2]);
    }
  }
  const double acoustic = cs * sqrt(1.0 / (d[0] * d[0]) + 1.0 / (d[1] * d[1]) + 1.0 / (d[2] * d[2]));
  const double convective = un[0] / d[0] + un[1] / d[1] + un[2] / d[2];
  m[0] = fmax(m[0], acoustic);
  m[1] = fmax(m[1], convective);
  m[2] = fmax(m[2], acoustic + convective);
}

// one grid row per block, its CTAs striding over the block's interior cells
// (a few hundred CTAs in all, so the atomics stay few); the sound speed of
// the state fromQ makes of Q (the cell's stored T as the iterative eos's
// starting guess when there is a state; with plane, the double flux's p off
// the cell's frozen plane); each CTA's maxima folded into out[0..2]
// (acoustic, convective, combined), which the caller zeroed.  A NaN cell is
// passed over, as fmax passes it.
template <int NS, bool RG>
__global__ void __launch_bounds__(256, RG ? 2 : 3) k_cflmax(const BlockDev *__restrict__ blks, int b, const double *__restrict__ Qall,
                         const double *__restrict__ stall, const double *__restrict__ met, double *out,
                         const int plane = 0) {
  const BlockDev &B = blks[b + blockIdx.y];
  const long long n = (long long)B.nx * B.ny * B.nz;
  double m[3] = {0.0, 0.0, 0.0};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    cfl_cell<NS, RG>(B, t, Qall, stall, met, plane, m);
  // the warp's maxima, then the CTA's, then one atomic per slot
  __shared__ double red[3][32];
#pragma unroll
  for (int q = 0; q < 3; q++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m[q] = fmax(m[q], __shfl_xor_sync(0xffffffffu, m[q], o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 3; q++) red[q][warp] = m[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      double x = lane < nwarps ? red[q][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
      if (lane == 0) cfl_atomic_max(out + q, x);
    }
  }
}

}  // namespace pgb
