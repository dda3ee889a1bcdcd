// The fused stage for blocks with uniform metrics: every face's area vector
// along its own axis, the inverse Jacobian diagonal and the cells evenly
// spaced (checked by the host on the block's own metric arrays).
//
// Same arithmetic as the general fused kernel, with the terms the uniform
// metrics make exactly zero left out: an off-axis area component, an
// off-diagonal of the inverse Jacobian, an off-axis damping or extrapolation
// distance.  Each dropped term is a product with an exact zero, so only the
// sign of a zero result can differ.  Two further choices, each a few ulp:
// the face velocities of kepaec (Q[1..3] / Q[0]) and of the viscous flux
// (Q[1..3] * rhoinv) are the one quotient, and the central differences of
// the gradients are of those quotients (the reference forms
// (Q+ rho- - Q- rho+) / (rho+ rho-), dqdxyz.mako:8-15).
//
// Layout of the work: a CTA of 256 threads, one thread per column of the
// tile and its one-cell ring (R1).  A column's cell values come from a
// shared plane; what a thread computes for its own column it keeps:
//   step k:  i- and j-faces below its cell at plane k (its low faces) into
//            shared; the loads of plane k+3 issued; plane k+2's values formed
//            from the loads of the step before; the gradients of plane k+1;
//            the k-face between k and k+1; dQ, combines and stores for the
//            tile's cells of plane k.
//
// Where a tile's ring or a plane beyond its block's k ends lies past a face,
// the cell comes either from the block's halo, filled by a launch before the
// stage, or (a.pull) straight from the neighbouring block's own cells, with
// no fill: every face of the case joined low face to high face in the
// identity orientation, unrotated, both blocks at least NG cells thick.  The
// block a cell comes from is the one a halo cell's source is located in
// (across i first, then j, then k), so the values, and the results, are the
// fill's to the bit.  Each thread works out its two cells' sources at tile
// start: the planes inside the block in registers, the planes below and
// above it in shared memory.
//
// Measured and set aside: one barrier a plane, with three plane slots, two
// gradient planes and two face-flux planes standing in for the second (the
// gradients of plane k+1 formed before the barrier, plane k+3's values after
// it): 210 registers and 212.7 KB of shared memory, the same results, but
// 0.294-0.336 ms a stage of the 27-block 128^3 TGV against 0.287-0.295 ms.
// The tile's warps carry every face and the k-face chain; moving the
// gradients ahead of the barrier lengthened their work before it more than
// the barrier it saved cost.
#pragma once
#include "fused.cuh"

namespace pgb {

constexpr int F2_THREADS = 256;
// cell values kept in shared memory per plane
enum { P_RHO = 0, P_U, P_V, P_W, P_T, P_E, P_N };

struct CellP {
  double rho, u, v, w, T, e;
};

__device__ __forceinline__ CellP prim_of(const double q0, const double q1, const double q2, const double q3,
                                         const double q4) {
  CellP c;
  const double ri = 1.0 / q0;
  c.rho = q0;
  c.e = (q4 - 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) * ri) * ri;
  c.T = quot(c.e - kSp.h2981, kSp.cv1, kSp.cvinv1);
  c.u = quot(q1, q0, ri);
  c.v = quot(q2, q0, ri);
  c.w = quot(q3, q0, ri);
  return c;
}

// One face of axis AX on uniform metrics: kepaec plus, with VISC, the
// single-species viscous rows, each with the zero-metric terms dropped.
// gL, gR: the two cells' gradients, rows u, v, w, T, 3 wide.
template <int AX, bool VISC>
__device__ __forceinline__ void face_u(const BlockDev &B, const CellP &L, const CellP &R, const double *gL,
                                       const double *gR, double *F) {
  const double S = B.S[AX];
  const double pL = L.rho * kSp.R1 * L.T, pR = R.rho * kSp.R1 * R.T;
  const double thL = kSp.th1 * L.T, thR = kSp.th1 * R.T;
  // kepaec.mako:3-17 with S = S e_AX
  const double uf = 0.5 * (R.u + L.u), vf = 0.5 * (R.v + L.v), wf = 0.5 * (R.w + L.w);
  const double ua = AX == 0 ? uf : AX == 1 ? vf : wf;
  const double U = S * ua;
  const double pf = 0.5 * (pR + pL);
  const double rho = 0.5 * (R.rho + L.rho);
  const double C = rho * U;
  F[0] = C;
  F[1] = AX == 0 ? C * uf + pf * S : C * uf;
  F[2] = AX == 1 ? C * vf + pf * S : C * vf;
  F[3] = AX == 2 ? C * wf + pf * S : C * wf;
  const double Kj = C * 0.5 * (R.u * L.u + R.v * L.v + R.w * L.w);
  const double uRa = AX == 0 ? R.u : AX == 1 ? R.v : R.w;
  const double uLa = AX == 0 ? L.u : AX == 1 ? L.v : L.w;
  const double Pj = 0.5 * (pL * (uRa * S) + pR * (uLa * S));
  const double ef = 2.0 * thL * thR / (thL + thR) + 0.5 * ((L.e - thL) + (R.e - thR));
  F[4] = ef * C + Kj + Pj;
  if constexpr (VISC) {
    // alpha-damping.mako:29-58 with the normal along AX
    const double mu = kSp.mu1, kappa = kSp.kappa1;
    const double lambda = 0.0 - 2.0 / 3.0 * mu;
    const double damp = B.damp[AX], xL = B.xL[AX], xR = B.xR[AX];
    // the face gradient of a row: the axis component damped toward the jump,
    // the others the sides' mean
    auto row = [&](const double phiL, const double phiR, const double *gl, const double *gr, double &ga, double &gb,
                   double &gc) {
      const double wl = phiL + gl[AX] * xL;
      const double wr = phiR + gr[AX] * xR;
      const double jump = wr - wl;
      ga = 0.5 * (gr[AX] + gl[AX]) + damp * jump;
      constexpr int B1 = (AX + 1) % 3, B2 = (AX + 2) % 3;
      gb = 0.5 * (gr[B1] + gl[B1]);
      gc = 0.5 * (gr[B2] + gl[B2]);
    };
    double d[3][3];  // d[row][direction]: du/dx ...
    {
      double a, b, c;
      row(L.u, R.u, gL + 0, gR + 0, a, b, c);
      d[0][AX] = a, d[0][(AX + 1) % 3] = b, d[0][(AX + 2) % 3] = c;
      row(L.v, R.v, gL + 3, gR + 3, a, b, c);
      d[1][AX] = a, d[1][(AX + 1) % 3] = b, d[1][(AX + 2) % 3] = c;
      row(L.w, R.w, gL + 6, gR + 6, a, b, c);
      d[2][AX] = a, d[2][(AX + 1) % 3] = b, d[2][(AX + 2) % 3] = c;
    }
    const double div = d[0][0] + d[1][1] + d[2][2];
    // the stress row of the face normal: tau[AX][m]
    double t0, t1, t2;
    if constexpr (AX == 0) {
      t0 = -2.0 * mu * d[0][0] - lambda * div;  // txx
      t1 = -mu * (d[1][0] + d[0][1]);           // txy
      t2 = -mu * (d[2][0] + d[0][2]);           // txz
    } else if constexpr (AX == 1) {
      t0 = -mu * (d[1][0] + d[0][1]);           // txy
      t1 = -2.0 * mu * d[1][1] - lambda * div;  // tyy
      t2 = -mu * (d[2][1] + d[1][2]);           // tyz
    } else {
      t0 = -mu * (d[2][0] + d[0][2]);           // txz
      t1 = -mu * (d[2][1] + d[1][2]);           // tyz
      t2 = -2.0 * mu * d[2][2] - lambda * div;  // tzz
    }
    F[1] += t0 * S;
    F[2] += t1 * S;
    F[3] += t2 * S;
    const double wlT = L.T + gL[9 + AX] * xL;
    const double wrT = R.T + gR[9 + AX] * xR;
    const double dTa = 0.5 * (gR[9 + AX] + gL[9 + AX]) + damp * (wrT - wlT);
    const double heatflux = -kappa * (dTa * S);
    const double f4 = (uf * t0 + vf * t1 + wf * t2) * S + heatflux;
    F[4] += f4;
  }
}

// the gradient rows u, v, w, T of a cell from its six neighbours' values
// (dqdxyz.mako:16-41 on a diagonal inverse Jacobian)
__device__ __forceinline__ void grad_u(const BlockDev &B, const CellP &xm, const CellP &xp, const CellP &ym,
                                       const CellP &yp, const CellP &zm, const CellP &zp, double *g) {
  const double Jx = B.Jd[0], Jy = B.Jd[1], Jz = B.Jd[2];
  g[0] = 0.5 * (xp.u - xm.u) * Jx, g[1] = 0.5 * (yp.u - ym.u) * Jy, g[2] = 0.5 * (zp.u - zm.u) * Jz;
  g[3] = 0.5 * (xp.v - xm.v) * Jx, g[4] = 0.5 * (yp.v - ym.v) * Jy, g[5] = 0.5 * (zp.v - zm.v) * Jz;
  g[6] = 0.5 * (xp.w - xm.w) * Jx, g[7] = 0.5 * (yp.w - ym.w) * Jy, g[8] = 0.5 * (zp.w - zm.w) * Jz;
  g[9] = 0.5 * (xp.T - xm.T) * Jx, g[10] = 0.5 * (yp.T - ym.T) * Jy, g[11] = 0.5 * (zp.T - zm.T) * Jz;
}

// cp.async (sm_80 and later): an 8-byte copy global -> shared that does not
// hold a register while in flight; groups complete in order
__device__ __forceinline__ void cp8(double *dst, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Shared memory of the uniform kernel, laid out for tiles of at most TW x TH
// cells (the layout's extents are compile-time, so every neighbour and field
// offset is an immediate; a tile may be smaller): P[2][LN2][P_N] two planes of
// cell values, a cell's six contiguous (48 bytes: three 16-byte loads, no two
// lanes of a quarter warp on one bank), G[LN1][GS] one plane of gradients,
// a cell's twelve contiguous in a record of GS (14 doubles, for the same
// reason), Fi[5][LN1], Fj[5][LN1]
// low-face fluxes, raw[3][5][NT + LNR] the Q copies of three planes in
// flight, pre[3][2][5][LNT] the combines' registers of three planes, and the
// sources of a thread's two fetched cells in the planes below and above the
// block (those inside it a thread keeps in registers): src[2][NT + LNR]
// pointers to the source cell's plane 0, then vol[2][NT + LNR] and
// plane[2][NT + LNR] its block's component and plane strides.
template <int NT, int TW, int TH>
struct F2L {
  static constexpr int LW1 = TW + 2, LH1 = TH + 2, LN1 = LW1 * LH1;
  static constexpr int LW2 = TW + 4, LN2 = LW2 * (TH + 4), LNR = 2 * (TW + TH), LNT = TW * TH;
  static constexpr int RAW = 5 * (NT + LNR), PRE = 2 * 5 * LNT, SRC = 2 * (NT + LNR);
  static constexpr int GS = 14;  // a gradient record: twelve values and two of padding
  static_assert(LN1 <= NT, "the tile and its ring fit the CTA");
  static_assert(LNR <= NT, "the outer ring fits the CTA");
  __host__ __device__ static constexpr size_t doubles(bool visc) {
    return (size_t)2 * P_N * LN2 + (visc ? GS * LN1 : 0) + 10 * LN1 + 3 * RAW + 3 * PRE + 2 * SRC;
  }
};

template <bool VISC, int NT, int MINB, int TW, int TH>
__global__ void __launch_bounds__(NT, MINB) k_fused2(const FusedArgs a) {
  using L = F2L<NT, TW, TH>;
  constexpr int LW1 = L::LW1, LN1 = L::LN1, LW2 = L::LW2, LN2 = L::LN2, LNR = L::LNR, LNT = L::LNT;
  extern __shared__ double smem[];
  __shared__ int s_tile;
  const int tid = threadIdx.x;
  double *P = smem;
  double *G = P + 2 * P_N * LN2;
  double *Fi = G + (VISC ? L::GS * LN1 : 0);
  double *Fj = Fi + 5 * LN1;
  double *raw = Fj + 5 * LN1;  // [3][5][NT] own cells then [5][LNR] ring cells, per slot
  double *pre = raw + 3 * L::RAW;  // [3][2][5][LNT]
  const double **src = reinterpret_cast<const double **>(pre + 3 * L::PRE);  // [2][NT + LNR]
  int *svol = reinterpret_cast<int *>(src + L::SRC), *splane = svol + L::SRC;
  for (;;) {
    if (tid == 0) s_tile = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int t = s_tile;
    __syncthreads();
    if (t >= a.ntiles) return;
    const TileDev T = a.tiles[t];
    const BlockDev &B = a.blks[T.blk];
    const int tw = T.tw, th = T.th;
    const int W1 = tw + 2, H1 = th + 2, N1 = W1 * H1;
    const int nring = 2 * (tw + th);
    const int v = (int)B.vol;
    const int sJ = B.X, sK = B.X * B.Y;
    const bool col = tid < N1;
    // the columns in warp order: the tile's first, then the ring's high edges
    // (the i-faces of its last column and the j-faces of its top row are the
    // tile's), then the rest of the ring, which has no face the tile needs,
    // so whole warps of it skip the face pass
    int ii = 0, jj = 0;
    {
      int q = tid;
      if (q < tw * th) ii = q % tw + 1, jj = q / tw + 1;
      else if ((q -= tw * th) < th) ii = tw + 1, jj = q + 1;
      else if ((q -= th) < tw) ii = q + 1, jj = th + 1;
      else if ((q -= tw) < th) ii = 0, jj = q + 1;
      else if ((q -= th) < tw) ii = q + 1, jj = 0;
      else if ((q -= tw) < 4) ii = (q & 1) ? tw + 1 : 0, jj = (q & 2) ? th + 1 : 0;
    }
    const bool needi = col && jj >= 1 && jj <= th && ii >= 1;
    const bool needj = col && ii >= 1 && ii <= tw && jj >= 1;
    const int c1 = ii + LW1 * jj;
    const int c2 = (ii + 1) + LW2 * (jj + 1);
    const bool tile = col && ii >= 1 && ii <= tw && jj >= 1 && jj <= th;
    const int tc = (ii - 1) + tw * (jj - 1);  // this tile cell's index, for the combine staging
    const bool ring_corner = (ii == 0 || ii == W1 - 1) && (jj == 0 || jj == H1 - 1);
    const bool gcol = col && !ring_corner;
    int r2 = -1, x2 = 0, y2 = 0;
    if (tid < nring) {
      int q = tid;
      if (q < th) x2 = 0, y2 = q + 2;
      else if ((q -= th) < th) x2 = tw + 3, y2 = q + 2;
      else if ((q -= th) < tw) x2 = q + 2, y2 = 0;
      else x2 = (q - tw) + 2, y2 = th + 3;
      r2 = x2 + LW2 * y2;
    }
    const int o1 = (T.j0 + jj + 1) * sJ + (T.i0 + ii + 1);
    // where each of this thread's fetched cells comes from, per k region:
    // the block's own cell (its halo beyond a face) or, when the stage pulls,
    // the cell of the block one step across each face it lies past (the
    // block a halo cell's source is located in, i first, then j, then k).
    // The planes inside the block (region 1) come back in q, sv, sk; those
    // below and above it (regions 0, 2) go to entry e of the shared table:
    // tid for the column, NT + tid for the outer ring cell.
    const double *Rq = a.R[a.qin];
    auto source_of = [&](int I, int J, int e, const double *&q, int &sv, int &sk) {
      const int di = I < 0 ? -1 : I < B.nx ? 0 : 1, dj = J < 0 ? -1 : J < B.ny ? 0 : 1;
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const int sb = a.pull ? a.nbr27[27 * T.blk + 9 * r + 3 * (dj + 1) + di + 1] : T.blk;
        const BlockDev &S = a.blks[sb];
        int i = I, j = J, dk = 0;
        if (a.pull) {
          i = di < 0 ? I + S.nx : di > 0 ? I - B.nx : I;
          j = dj < 0 ? J + S.ny : dj > 0 ? J - B.ny : J;
          dk = r == 0 ? S.nz : r == 2 ? -B.nz : 0;
        }
        const int plane = S.X * S.Y;
        const double *at = Rq + 5 * S.cv + (long long)(dk + NG) * plane + (j + NG) * S.X + (i + NG);
        if (r == 1) {
          q = at, sv = (int)S.vol, sk = plane;
        } else {
          const int x = (r >> 1) * (NT + LNR) + e;
          src[x] = at, svol[x] = (int)S.vol, splane[x] = plane;
        }
      }
    };
    const double *qc = nullptr, *qr = nullptr;
    int vc = 0, kc = 0, vr = 0, kr = 0;
    if (col) source_of(T.i0 + ii - 1, T.j0 + jj - 1, tid, qc, vc, kc);
    if (r2 >= 0) source_of(T.i0 + x2 - 2, T.j0 + y2 - 2, NT + tid, qr, vr, kr);
    auto slot = [](int p) { return p & 1; };
    auto ring3 = [](int p) { return (p + 6) % 3; };
    auto getP = [&](int s, int r) {
      const double2 *Ps = reinterpret_cast<const double2 *>(P + s * P_N * LN2 + P_N * r);
      const double2 a = Ps[0], b = Ps[1], d = Ps[2];
      CellP c;
      c.rho = a.x, c.u = a.y, c.v = b.x, c.w = b.y, c.T = d.x, c.e = d.y;
      return c;
    };
    auto putP = [&](int s, int r, const CellP &c) {
      double2 *Ps = reinterpret_cast<double2 *>(P + s * P_N * LN2 + P_N * r);
      Ps[0] = make_double2(c.rho, c.u), Ps[1] = make_double2(c.v, c.w), Ps[2] = make_double2(c.T, c.e);
    };
    // plane p's Q copies for this thread's cells, into raw slot p mod 3
    const int nzb = B.nz;
    auto fetch = [&](int p) {
      double *rs = raw + ring3(p) * L::RAW;
      const bool inside = p >= 0 && p < nzb;
      const int r = (p < 0 ? 0 : 1) * (NT + LNR);
      if (col) {
        const double *q = inside ? qc + p * kc : src[r + tid] + p * splane[r + tid];
        const int sv = inside ? vc : svol[r + tid];
#pragma unroll
        for (int l = 0; l < 5; l++) cp8(rs + l * NT + tid, q + l * sv);
      }
      if (r2 >= 0) {
        const double *q = inside ? qr + p * kr : src[r + NT + tid] + p * splane[r + NT + tid];
        const int sv = inside ? vr : svol[r + NT + tid];
#pragma unroll
        for (int l = 0; l < 5; l++) cp8(rs + 5 * NT + l * LNR + tid, q + l * sv);
      }
    };
    // plane p's combine registers for a tile cell, into pre slot p mod 3
    const long long cbase = 5 * B.cv + o1;
    const double *pre0 = a.prep[0] ? a.prep[0] + cbase : nullptr;
    const double *pre1 = a.prep[1] ? a.prep[1] + cbase : nullptr;
    auto fetch_pre = [&](int p) {
      if (!tile) return;
      double *ps = pre + ring3(p) * L::PRE + tc;
      const int z = (p + NG) * sK;
      if (pre0) {
#pragma unroll
        for (int l = 0; l < 5; l++) cp8(ps + l * LNT, pre0 + z + l * v);
      }
      if (pre1) {
#pragma unroll
        for (int l = 0; l < 5; l++) cp8(ps + (5 + l) * LNT, pre1 + z + l * v);
      }
    };
    // a slot no register fills holds zeros, so its zero weight adds nothing
    if (!pre1 && tile)
      for (int q = 0; q < 3; q++)
#pragma unroll
        for (int l = 0; l < 5; l++) pre[q * L::PRE + (5 + l) * LNT + tc] = 0.0;
    if (!pre0 && tile)
      for (int q = 0; q < 3; q++)
#pragma unroll
        for (int l = 0; l < 5; l++) pre[q * L::PRE + l * LNT + tc] = 0.0;
    auto own_raw = [&](int p) {
      const double *rs = raw + ring3(p) * L::RAW + tid;
      return prim_of(rs[0 * NT], rs[1 * NT], rs[2 * NT], rs[3 * NT], rs[4 * NT]);
    };
    auto ring_raw = [&](int p) {
      const double *rs = raw + ring3(p) * L::RAW + 5 * NT + tid;
      return prim_of(rs[0 * LNR], rs[1 * LNR], rs[2 * LNR], rs[3 * LNR], rs[4 * LNR]);
    };
    auto putG = [&](const double *g) {
#pragma unroll
      for (int q = 0; q < 12; q += 2)
        reinterpret_cast<double2 *>(G + L::GS * c1)[q / 2] = make_double2(g[q], g[q + 1]);
    };
    auto grad_col = [&](int s, const CellP &below, const CellP &above, double *g) {
      grad_u(B, getP(s, c2 - 1), getP(s, c2 + 1), getP(s, c2 - LW2), getP(s, c2 + LW2), below, above, g);
    };

    const int k0 = T.k0, k1 = T.k1;
    // prelude: the copies of planes k0-2 .. k0 go out together; each is
    // turned into cell values as it lands while the next copies go out
    CellP pm2{}, pm1{}, p0{}, p1{};
    fetch(k0 - 2);
    cp_commit();
    fetch(k0 - 1);
    cp_commit();
    fetch(k0);
    cp_commit();
    cp_wait<2>();
    if (col) pm2 = own_raw(k0 - 2);
    fetch(k0 + 1);
    cp_commit();
    cp_wait<2>();
    if (col) putP(slot(k0 - 1), c2, pm1 = own_raw(k0 - 1));
    if (r2 >= 0) putP(slot(k0 - 1), r2, ring_raw(k0 - 1));
    fetch(k0 + 2);
    fetch_pre(k0);
    cp_commit();
    cp_wait<2>();
    if (col) putP(slot(k0), c2, p0 = own_raw(k0));
    if (r2 >= 0) putP(slot(k0), r2, ring_raw(k0));
    if (k0 + 3 <= k1 + 1) fetch(k0 + 3);
    if (k0 + 1 < k1) fetch_pre(k0 + 1);
    cp_commit();
    __syncthreads();
    double gbelow[12];
    if (VISC && tile) grad_col(slot(k0 - 1), pm2, p0, gbelow);
    cp_wait<2>();
    __syncthreads();
    if (col) putP(slot(k0 + 1), c2, p1 = own_raw(k0 + 1));
    if (r2 >= 0) putP(slot(k0 + 1), r2, ring_raw(k0 + 1));
    __syncthreads();
    double Fk[5];
    {
      double g0[12];
      if (VISC && gcol) {
        grad_col(slot(k0), pm1, p1, g0);
        putG(g0);
      }
      if (tile) face_u<2, VISC>(B, pm1, p0, gbelow, g0, Fk);
    }
    __syncthreads();
    const double dt = *a.dt;
    const double c00 = a.cw[0][0], c01 = a.cw[0][1], c02 = a.cw[0][2] * dt;
    const double c10 = a.cw[1][0], c11 = a.cw[1][1], c12 = a.cw[1][2] * dt, c13 = a.cw[1][3];
    double *const out0 = a.outp[0], *const out1 = a.outp[1];
    const bool wr0 = a.write[0] && out0, wr1 = a.write[1] && out1;

    // in flight at the top of step k: {plane k+2, combine registers of k},
    // {plane k+3, combine registers of k+1}
    for (int k = k0; k < k1; k++) {
      const int s0 = slot(k), s1 = slot(k + 1);
      // 0. the copies of plane k+4 and of plane k+2's combine registers go
      //    out: their slots held plane k+1 and k-1, used up last step
      if (k + 4 <= k1 + 1) fetch(k + 4);
      if (k + 2 < k1) fetch_pre(k + 2);
      cp_commit();
      // 1. this column's low i and j faces at plane k, both in one straight
      //    run so their arithmetic interleaves; a ring column on the tile's
      //    high edges computes both and keeps the one the tile needs, the
      //    rest of the ring (whole warps of it) none
      if (needi || needj) {
        const int li = ii >= 1 ? 1 : 0, lj = jj >= 1 ? LW1 : 0;
        const int li2 = ii >= 1 ? 1 : 0, lj2 = jj >= 1 ? LW2 : 0;
        double Fa[5], Fb[5], gli[12], glj[12], gr[12];
        if (VISC) {
          const double2 *Gi = reinterpret_cast<const double2 *>(G + L::GS * (c1 - li));
          const double2 *Gj = reinterpret_cast<const double2 *>(G + L::GS * (c1 - lj));
          const double2 *Gr = reinterpret_cast<const double2 *>(G + L::GS * c1);
#pragma unroll
          for (int q = 0; q < 6; q++) {
            const double2 x = Gi[q], y = Gj[q], z = Gr[q];
            gli[2 * q] = x.x, gli[2 * q + 1] = x.y, glj[2 * q] = y.x, glj[2 * q + 1] = y.y;
            gr[2 * q] = z.x, gr[2 * q + 1] = z.y;
          }
        }
        const CellP me = getP(s0, c2);
        face_u<0, VISC>(B, getP(s0, c2 - li2), me, gli, gr, Fa);
        face_u<1, VISC>(B, getP(s0, c2 - lj2), me, glj, gr, Fb);
        if (needi) {
#pragma unroll
          for (int l = 0; l < 5; l++) Fi[l * LN1 + c1] = Fa[l];
        }
        if (needj) {
#pragma unroll
          for (int l = 0; l < 5; l++) Fj[l * LN1 + c1] = Fb[l];
        }
      }
      // 2. plane k+2 and plane k's combine registers have landed
      cp_wait<2>();
      CellP p2{}, p2r{};
      if (col) p2 = own_raw(k + 2);
      if (r2 >= 0) p2r = ring_raw(k + 2);
      __syncthreads();
      // 3. the gradients of plane k+1, the k face above k, dQ and the combines
      const CellP pk = col ? getP(s0, c2) : CellP{};
      const CellP pk1 = col ? getP(s1, c2) : CellP{};
      double gup[12];
      if (VISC && gcol) grad_col(s1, pk, p2, gup);
      if (tile) {
        double Fkh[5], gk[12];
        if (VISC) {
          const double2 *Gc = reinterpret_cast<const double2 *>(G + L::GS * c1);
#pragma unroll
          for (int q = 0; q < 6; q++) {
            const double2 x = Gc[q];
            gk[2 * q] = x.x, gk[2 * q + 1] = x.y;
          }
        } else {
#pragma unroll
          for (int q = 0; q < 12; q++) gk[q] = 0.0;
        }
        face_u<2, VISC>(B, pk, pk1, gk, gup, Fkh);
        const double dJ = B.detJinv;
        double dQ[5];
#pragma unroll
        for (int l = 0; l < 5; l++)
          dQ[l] = (Fi[l * LN1 + c1] + Fj[l * LN1 + c1] + Fk[l] - Fi[l * LN1 + c1 + 1] - Fj[l * LN1 + c1 + LW1] - Fkh[l]) * dJ;
        // the combines in their fixed form (no branch, no register lookup)
        const long long at = cbase + (k + NG) * sK;
        const double *pk3 = pre + ring3(k) * L::PRE + tc;
#pragma unroll
        for (int l = 0; l < 5; l++) {
          const double p0 = pk3[l * LNT], p1 = pk3[(5 + l) * LNT];
          const double o0 = c00 * p0 + c01 * p1 + c02 * dQ[l];
          const double o1v = c10 * p0 + c11 * p1 + c12 * dQ[l] + c13 * o0;
          if (wr0) out0[at + l * v] = o0;
          if (wr1) out1[at + l * v] = o1v;
        }
#pragma unroll
        for (int l = 0; l < 5; l++) Fk[l] = Fkh[l];
      }
      // 4. plane k+2 takes plane k's slot, the k+1 gradients plane k's
      if (col) putP(s0, c2, p2);
      if (r2 >= 0) putP(s0, r2, p2r);
      if (VISC && gcol) putG(gup);
      __syncthreads();
    }
    cp_wait<0>();
  }
}

template <int NT, int TW, int TH>
inline size_t fused2_smem(bool visc) {
  return sizeof(double) * F2L<NT, TW, TH>::doubles(visc);
}

}  // namespace pgb
