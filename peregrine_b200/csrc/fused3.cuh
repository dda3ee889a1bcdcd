// The fused stage for blocks with uniform metrics, warp-specialised: the
// same arithmetic as k_fused2 (face_u, grad_u, prim_of, the fixed combine
// form), its work spread over sixteen warps of at most 128 registers a
// thread, with one barrier per plane.
//
// A CTA takes a tile of at most TW x TH cells and marches it along k, one
// pass per plane.  Its warps come in four roles of four warps, each item of
// a role one thread:
//   role 0  the gradients of plane k+1 at the tile's cells;
//   role 1  the i-faces of plane k;      role 2  its j-faces;
//   role 3  the k-face between planes k-1 and k at the tile's cells;
// and the threads of roles 0-2 take at most one more task each: the dQ and
// combines of a tile cell at plane k-2, the cell values of plane k+3 at a
// cell of the tile and its two-cell ring (from the Q copies the same thread
// fetched a pass before), or the gradients of plane k+1 at a cell of the
// one-cell ring.  Everything a pass reads, an earlier pass wrote: five
// planes of cell values, three of gradients, of face fluxes and of the
// combines' registers, two of Q copies in flight.
#pragma once
#include "fused2.cuh"

namespace pgb {

template <int NT, int TW, int TH>
struct F3L {
  static constexpr int PW = TW + 4, NP = PW * (TH + 4);  // cell values: the tile and its two-cell ring
  static constexpr int GW = TW + 2, NG1 = GW * (TH + 2); // gradients: the tile and its one-cell ring
  static constexpr int FIW = TW + 1, NFI = FIW * TH;     // i-faces
  static constexpr int NFJ = TW * (TH + 1);              // j-faces
  static constexpr int NC = TW * TH;                     // tile cells
  static constexpr int NR = 2 * (TW + TH);               // one-cell ring less its corners
  static constexpr int ROLE = 128;                       // threads of each role's four warps
  static_assert(NT == 512, "sixteen warps: four roles of four");
  static_assert(NC <= ROLE && NFI <= ROLE && NFJ <= ROLE, "each role's items fit its warps");
  static_assert(NC + NP + NR <= 3 * ROLE, "one extra task a thread of roles 0-2");
  // offsets in doubles
  static constexpr int oP = 0;
  static constexpr int oG = oP + 5 * P_N * NP;
  template <bool V>
  __host__ __device__ static constexpr int oFi() { return oG + (V ? 3 * 12 * NG1 : 0); }
  template <bool V>
  __host__ __device__ static constexpr int oFj() { return oFi<V>() + 3 * 5 * NFI; }
  template <bool V>
  __host__ __device__ static constexpr int oFk() { return oFj<V>() + 3 * 5 * NFJ; }
  template <bool V>
  __host__ __device__ static constexpr int oRaw() { return oFk<V>() + 3 * 5 * NC; }
  template <bool V>
  __host__ __device__ static constexpr int oPre() { return oRaw<V>() + 2 * 5 * NP; }
  template <bool V>
  __host__ __device__ static constexpr int total() { return oPre<V>() + 3 * 10 * NC; }
};

template <bool VISC, int NT, int MINB, int TW, int TH>
__global__ void __launch_bounds__(NT, MINB) k_fused3(const FusedArgs a) {
  using L = F3L<NT, TW, TH>;
  constexpr int PW = L::PW, NP = L::NP, GW = L::GW, NG1 = L::NG1, FIW = L::FIW, NFI = L::NFI, NFJ = L::NFJ,
                NC = L::NC, ROLE = L::ROLE;
  extern __shared__ double smem[];
  __shared__ int s_tile;
  const int tid = threadIdx.x;
  double *const P = smem + L::oP;
  double *const G = smem + L::oG;
  double *const Fi = smem + L::template oFi<VISC>();
  double *const Fj = smem + L::template oFj<VISC>();
  double *const Fk = smem + L::template oFk<VISC>();
  double *const raw = smem + L::template oRaw<VISC>();
  double *const pre = smem + L::template oPre<VISC>();
  const int role = tid / ROLE;
  const int ridx = tid - role * ROLE;
  // slots of plane p in rings of five, three and two
  auto s5 = [](int p) { return (p + 15) % 5; };
  auto s3 = [](int p) { return (p + 6) % 3; };
  auto getP = [&](int p, int r) {
    const double *Ps = P + s5(p) * P_N * NP + r;
    CellP c;
    c.rho = Ps[P_RHO * NP], c.u = Ps[P_U * NP], c.v = Ps[P_V * NP];
    c.w = Ps[P_W * NP], c.T = Ps[P_T * NP], c.e = Ps[P_E * NP];
    return c;
  };
  auto putP = [&](int p, int r, const CellP &c) {
    double *Ps = P + s5(p) * P_N * NP + r;
    Ps[P_RHO * NP] = c.rho, Ps[P_U * NP] = c.u, Ps[P_V * NP] = c.v;
    Ps[P_W * NP] = c.w, Ps[P_T * NP] = c.T, Ps[P_E * NP] = c.e;
  };
  // a cell's gradients at plane p from its four in-plane neighbours' cell
  // values and its two k-neighbours', into gradient slot p
  auto grad_put = [&](const BlockDev &B, int p, int r, int gi) {
    double g[12];
    grad_u(B, getP(p, r - 1), getP(p, r + 1), getP(p, r - PW), getP(p, r + PW), getP(p - 1, r), getP(p + 1, r), g);
    double *Gs = G + s3(p) * 12 * NG1 + gi;
#pragma unroll
    for (int q = 0; q < 12; q++) Gs[q * NG1] = g[q];
  };
  auto getG = [&](int p, int gi, double *g) {
    const double *Gs = G + s3(p) * 12 * NG1 + gi;
#pragma unroll
    for (int q = 0; q < 12; q++) g[q] = Gs[q * NG1];
  };

  for (;;) {
    if (tid == 0) s_tile = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int t = s_tile;
    __syncthreads();
    if (t >= a.ntiles) return;
    const TileDev T = a.tiles[t];
    const BlockDev &B = a.blks[T.blk];
    const int tw = T.tw, th = T.th, k0 = T.k0, k1 = T.k1;
    const int v = (int)B.vol;
    const int sJ = B.X, sK = B.X * B.Y;
    const double *Q = a.R[a.qin] + 5 * B.cv;
    // a cell (x, y) of the tile's frame, the tile's cells at 2..tw+1, 2..th+1:
    // its offset in a plane of the block's arrays and its index in the layouts
    auto goff = [&](int x, int y) { return (T.j0 + y) * sJ + (T.i0 + x); };
    auto pidx = [](int x, int y) { return x + PW * y; };
    auto gidx = [](int x, int y) { return (x - 1) + GW * (y - 1); };
    auto cidx = [](int x, int y) { return (x - 2) + TW * (y - 2); };

    // the role's item
    int rx = 0, ry = 0;
    bool ract = false;
    if ((role == 0 || role == 3) && ridx < tw * th) ract = true, rx = ridx % tw + 2, ry = ridx / tw + 2;
    if (role == 1 && ridx < (tw + 1) * th) ract = true, rx = ridx % (tw + 1) + 2, ry = ridx / (tw + 1) + 2;
    if (role == 2 && ridx < tw * (th + 1)) ract = true, rx = ridx % tw + 2, ry = ridx / tw + 2;
    const int rp = pidx(rx, ry);
    // the extra task of a thread of roles 0-2: role 0's threads (the light
    // gradients) take the dQ, the others the cell values and the ring's
    // gradients
    enum { X_NONE = 0, X_DQ, X_PRIM, X_RING };
    int xk = X_NONE, xx = 0, xy = 0;
    if (role < 3) {
      int m = tid;
      const int nc = tw * th, np = (tw + 4) * (th + 4), nr = 2 * (tw + th);
      if (m < nc) {
        xk = X_DQ, xx = m % tw + 2, xy = m / tw + 2;
      } else if ((m -= nc) < np) {
        xk = X_PRIM, xx = m % (tw + 4), xy = m / (tw + 4);
      } else if (VISC && (m -= np) < nr) {
        xk = X_RING;
        if (m < th) xx = 1, xy = m + 2;
        else if ((m -= th) < th) xx = tw + 2, xy = m + 2;
        else if ((m -= th) < tw) xx = m + 2, xy = 1;
        else xx = (m - tw) + 2, xy = th + 2;
      }
    }
    const int xo = goff(xx, xy), xp = pidx(xx, xy);
    // the prim task's Q copies of plane p into raw slot p mod 2
    auto fetch = [&](int p) {
      if (xk != X_PRIM) return;
      double *rs = raw + (p & 1) * 5 * NP + xp;
      const double *src = Q + (p + NG) * sK + xo;
#pragma unroll
      for (int l = 0; l < 5; l++) cp8(rs + l * NP, src + l * v);
    };
    auto prim = [&](int p) {
      if (xk != X_PRIM) return;
      const double *rs = raw + (p & 1) * 5 * NP + xp;
      putP(p, xp, prim_of(rs[0], rs[NP], rs[2 * NP], rs[3 * NP], rs[4 * NP]));
    };
    // the dQ task's combine registers of plane p into pre slot p mod 3
    const int xc = xk == X_DQ ? cidx(xx, xy) : 0;
    auto fetch_pre = [&](int p) {
      if (xk != X_DQ) return;
      double *ps = pre + s3(p) * 10 * NC + xc;
      const long long at = 5 * B.cv + xo + (long long)(p + NG) * sK;
      if (a.prep[0]) {
#pragma unroll
        for (int l = 0; l < 5; l++) cp8(ps + l * NC, a.prep[0] + at + (long long)l * v);
      }
      if (a.prep[1]) {
#pragma unroll
        for (int l = 0; l < 5; l++) cp8(ps + (5 + l) * NC, a.prep[1] + at + (long long)l * v);
      }
    };
    // a slot no register fills holds zeros, so its zero weight adds nothing
    if (xk == X_DQ) {
      for (int s = 0; s < 3; s++) {
#pragma unroll
        for (int l = 0; l < 5; l++) {
          if (!a.prep[0]) pre[s * 10 * NC + l * NC + xc] = 0.0;
          if (!a.prep[1]) pre[s * 10 * NC + (5 + l) * NC + xc] = 0.0;
        }
      }
    }

    // prelude: the cell values of planes k0-2 .. k0+2 and the gradients of
    // planes k0-1 and k0; the copies of plane k0+3 go out
    fetch(k0 - 2);
    fetch(k0 - 1);
    cp_commit();
    cp_wait<0>();
    prim(k0 - 2);
    prim(k0 - 1);
    fetch(k0);
    fetch(k0 + 1);
    cp_commit();
    cp_wait<0>();
    prim(k0);
    prim(k0 + 1);
    fetch(k0 + 2);
    cp_commit();
    cp_wait<0>();
    prim(k0 + 2);
    fetch(k0 + 3);
    cp_commit();
    __syncthreads();
    if (VISC) {
      if (role == 0 && ract) {
        grad_put(B, k0 - 1, rp, gidx(rx, ry));
        grad_put(B, k0, rp, gidx(rx, ry));
      }
      if (xk == X_RING) {
        grad_put(B, k0 - 1, xp, gidx(xx, xy));
        grad_put(B, k0, xp, gidx(xx, xy));
      }
    }
    __syncthreads();

    // pass k: the gradients of plane k+1, the i- and j-faces of plane k, the
    // k-face below it, the cell values of plane k+3 and the dQ of plane k-2
    for (int k = k0; k <= k1 + 1; k++) {
      // the copies of plane k+4 and of plane k's combine registers go out; those
      // of plane k+3, out since the last pass, land
      if (k + 4 <= k1 + 1) fetch(k + 4);
      if (k < k1) fetch_pre(k);
      cp_commit();
      cp_wait<1>();
      if (role == 0) {
        if (VISC && ract && k < k1) grad_put(B, k + 1, rp, gidx(rx, ry));
      } else if (role == 1) {
        if (ract && k < k1) {
          double gl[12], gr[12], F[5];
          if (VISC) getG(k, gidx(rx - 1, ry), gl), getG(k, gidx(rx, ry), gr);
          face_u<0, VISC>(B, getP(k, rp - 1), getP(k, rp), gl, gr, F);
          double *Fs = Fi + s3(k) * 5 * NFI + (rx - 2) + FIW * (ry - 2);
#pragma unroll
          for (int l = 0; l < 5; l++) Fs[l * NFI] = F[l];
        }
      } else if (role == 2) {
        if (ract && k < k1) {
          double gl[12], gr[12], F[5];
          if (VISC) getG(k, gidx(rx, ry - 1), gl), getG(k, gidx(rx, ry), gr);
          face_u<1, VISC>(B, getP(k, rp - PW), getP(k, rp), gl, gr, F);
          double *Fs = Fj + s3(k) * 5 * NFJ + (rx - 2) + TW * (ry - 2);
#pragma unroll
          for (int l = 0; l < 5; l++) Fs[l * NFJ] = F[l];
        }
      } else if (ract && k <= k1) {
        double gl[12], gr[12], F[5];
        if (VISC) getG(k - 1, gidx(rx, ry), gl), getG(k, gidx(rx, ry), gr);
        face_u<2, VISC>(B, getP(k - 1, rp), getP(k, rp), gl, gr, F);
        double *Fs = Fk + s3(k - 1) * 5 * NC + cidx(rx, ry);
#pragma unroll
        for (int l = 0; l < 5; l++) Fs[l * NC] = F[l];
      }
      if (k + 3 <= k1 + 1) prim(k + 3);
      if (VISC && xk == X_RING && k < k1) grad_put(B, k + 1, xp, gidx(xx, xy));
      if (xk == X_DQ && k >= k0 + 2) {
        // the weights and outputs read where they are used: a thread of
        // another task holds none of them
        const double dt = *a.dt, dJ = B.detJinv;
        const double c00 = a.cw[0][0], c01 = a.cw[0][1], c02 = a.cw[0][2] * dt;
        const double c10 = a.cw[1][0], c11 = a.cw[1][1], c12 = a.cw[1][2] * dt, c13 = a.cw[1][3];
        double *const out0 = a.outp[0], *const out1 = a.outp[1];
        const bool wr0 = a.write[0] && out0, wr1 = a.write[1] && out1;
        const int m = k - 2;
        const int fi = (xx - 2) + FIW * (xy - 2), fj = (xx - 2) + TW * (xy - 2);
        const double *Fis = Fi + s3(m) * 5 * NFI, *Fjs = Fj + s3(m) * 5 * NFJ;
        const double *Fkl = Fk + s3(m - 1) * 5 * NC + xc, *Fkh = Fk + s3(m) * 5 * NC + xc;
        const double *pk = pre + s3(m) * 10 * NC + xc;
        const long long at = 5 * B.cv + xo + (long long)(m + NG) * sK;
#pragma unroll
        for (int l = 0; l < 5; l++) {
          const double dQ = (Fis[l * NFI + fi] + Fjs[l * NFJ + fj] + Fkl[l * NC] - Fis[l * NFI + fi + 1] -
                             Fjs[l * NFJ + fj + TW] - Fkh[l * NC]) * dJ;
          const double p0 = pk[l * NC], p1 = pk[(5 + l) * NC];
          const double o0 = c00 * p0 + c01 * p1 + c02 * dQ;
          const double o1v = c10 * p0 + c11 * p1 + c12 * dQ + c13 * o0;
          if (wr0) out0[at + (long long)l * v] = o0;
          if (wr1) out1[at + (long long)l * v] = o1v;
        }
      }
      __syncthreads();
    }
    cp_wait<0>();
  }
}

template <int NT, int TW, int TH>
inline size_t fused3_smem(bool visc) {
  using L = F3L<NT, TW, TH>;
  return sizeof(double) * (visc ? L::template total<true>() : L::template total<false>());
}

}  // namespace pgb
