// The fused stage: the whole right-hand side and the Runge-Kutta combine of
// one stage in one persistent launch over every block of the case.
//
// It covers the calorically perfect single-species gas with the kepaec flux
// on the cells as they are, inviscid or with the alpha-damping viscous flux
// and constant transport: the reference's fromQ, transport, dqdxyz, flux
// (advective and diffusive, three axes), applyflux and combine kernels
// (peregrine/simulator/advecdiff/simulator.py:110-124,
//  peregrine/integrators/rungekutta.py:84-92), with each cell's state read
// from HBM once per stage and dQ never stored.
//
// Work: a queue of tiles, each a tw x th column of one block over a run of
// k planes; a CTA takes the next tile from an atomic counter until none are
// left.  A tile marches up k keeping three planes of cell values, two planes
// of gradients and one plane of face fluxes in shared memory:
//   plane k+2's cells are loaded (the tile plus two cells around it),
//   plane k+1's gradients are formed (the tile plus one cell around),
//   plane k's i and j faces and the k face above it are fluxed,
//   plane k's cells get dQ and the stage's combines.
// Each face flux is formed once and read by the two cells it joins.
#pragma once
#include "layout.cuh"
#include "physics.cuh"

namespace pgb {

constexpr int FUSED_THREADS = 128;
constexpr int MAXREGS = 6;

// the stage's combines, on physical registers: out = sum_n w[n] X[n], summed
// left to right, dt multiplying the last term when step is set.  A term's
// src is a physical register, -1 for this stage's dQ, -2 for the first
// combine's result at this cell; a combine that reads its own output has it
// as term 0 (the reference's wout * out).  write 0 drops a store no later
// stage reads.
struct FusedCombine {
  int out, nterms, step, write;
  int src[4];
  double w[4];
};

struct FusedArgs {
  const BlockDev *blks;
  const TileDev *tiles;
  int ntiles;
  unsigned int *counter;
  const double *met;
  double *R[MAXREGS];
  int qin;
  int ncomb;
  FusedCombine comb[2];
  // the same combines with each register term as a slot of the registers
  // the uniform kernel copies ahead (pre[slot] the physical register)
  int npre;
  int pre[3];
  FusedCombine combp[2];
  // the same combines as one fixed form the uniform kernel evaluates with no
  // branch: out0 = c[0][0] p0 + c[0][1] p1 + c[0][2] dt dQ, and
  // out1 = c[1][0] p0 + c[1][1] p1 + c[1][2] dt dQ + c[1][3] out0, summed in
  // that order, a missing term's weight zero (its register slot holds zeros);
  // p0, p1 the registers the stage reads (slots 0 and 1), in the order the
  // reference's combines name them
  double cw[2][4];
  double *outp[2];
  const double *prep[2];
  int write[2];
  const double *dt;
  // 1: the uniform kernel reads its tiles' ring and the planes beyond a
  // block's k ends from the neighbouring blocks' cells (every face joined,
  // unrotated, in the identity orientation, the neighbour at least NG cells
  // thick), and no halo fill precedes it; nbr27[27 b + q] is then the block
  // one step away from b along each axis, q = (dk + 1) 9 + (dj + 1) 3 + di + 1
  int pull;
  const int *nbr27;
};

// fields of a cell plane in shared memory
enum { A_Q0 = 0, A_Q1, A_Q2, A_Q3, A_T, A_RI, A_E, A_N };

// a quotient from the divisor's reciprocal, corrected by one residual
// (Markstein's division step: q = a y, r = a - q b, q + r y)
__device__ __forceinline__ double quot(const double a, const double b, const double y) {
  const double q = a * y;
  const double r = fma(-q, b, a);
  return fma(r, y, q);
}

template <bool VISC, bool UNIFORM>
__global__ void __launch_bounds__(FUSED_THREADS, 2) k_fused1(const FusedArgs a) {
  extern __shared__ double smem[];
  __shared__ int s_tile;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_tile = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int t = s_tile;
    __syncthreads();
    if (t >= a.ntiles) return;
    const TileDev T = a.tiles[t];
    const BlockDev &B = a.blks[T.blk];
    const int tw = T.tw, th = T.th;
    const int W2 = tw + 4, H2 = th + 4, N2 = W2 * H2;
    const int W1 = tw + 2, H1 = th + 2, N1 = W1 * H1;
    // shared layout: A[3][A_N][N2], G[2][12][N1], Fi[5][N1], Fj[5][N1]
    double *A = smem;
    double *G = A + 3 * A_N * N2;
    double *Fi = G + (VISC ? 2 * 12 * N1 : 0);
    double *Fj = Fi + 5 * N1;
    const long long v = B.vol;
    const long long sJ = B.X, sK = (long long)B.X * B.Y;
    const double *Q = a.R[a.qin] + 5 * B.cv;
    const double *M = a.met + M_NCOMP * B.cv;
    // full-array index of the tile's R2 origin at plane 0
    const int fi0 = T.i0, fj0 = T.j0;  // interior i0 - 2 + NG
    auto slot3 = [](int k) { return (k + 3) % 3; };
    auto slot2 = [](int k) { return (k + 2) % 2; };

    // plane p (interior index) into A slot: Q, T, rhoinv, e on the whole R2 region
    auto load_plane = [&](int p) {
      double *As = A + slot3(p) * A_N * N2;
      const long long zoff = (long long)(p + NG) * sK;
      for (int r = tid; r < N2; r += FUSED_THREADS) {
        const int ii = r % W2, jj = r / W2;
        const long long c = zoff + (long long)(fj0 + jj) * sJ + (fi0 + ii);
        const double q0 = __ldg(Q + c), q1 = __ldg(Q + v + c), q2 = __ldg(Q + 2 * v + c);
        const double q3 = __ldg(Q + 3 * v + c), q4 = __ldg(Q + 4 * v + c);
        const double ri = 1.0 / q0;
        const double e = (q4 - 0.5 * (q1 * q1 + q2 * q2 + q3 * q3) * ri) * ri;
        const double Tc = quot(e - kSp.h2981, kSp.cv1, kSp.cvinv1);
        As[A_Q0 * N2 + r] = q0;
        As[A_Q1 * N2 + r] = q1;
        As[A_Q2 * N2 + r] = q2;
        As[A_Q3 * N2 + r] = q3;
        As[A_T * N2 + r] = Tc;
        As[A_RI * N2 + r] = ri;
        As[A_E * N2 + r] = e;
      }
    };

    // gradients of plane p on R1 into G slot
    auto grad_plane = [&](int p) {
      if constexpr (VISC) {
        const double *Am = A + slot3(p - 1) * A_N * N2;
        const double *Ac = A + slot3(p) * A_N * N2;
        const double *Ap = A + slot3(p + 1) * A_N * N2;
        double *Gs = G + slot2(p) * 12 * N1;
        const long long zoff = (long long)(p + NG) * sK;
        for (int r = tid; r < N1; r += FUSED_THREADS) {
          const int ii = r % W1 + 1, jj = r / W1 + 1;
          const int c2 = ii + W2 * jj;
          const int xp = c2 + 1, xm = c2 - 1, yp = c2 + W2, ym = c2 - W2;
          double Jm[9];
          if constexpr (UNIFORM) {
            Jm[0] = B.Jd[0], Jm[4] = B.Jd[1], Jm[8] = B.Jd[2];
            Jm[1] = Jm[2] = Jm[3] = Jm[5] = Jm[6] = Jm[7] = 0.0;
          } else {
            const long long gc = zoff + (long long)(fj0 + jj) * sJ + (fi0 + ii);
#pragma unroll
            for (int q = 0; q < 9; q++) Jm[q] = __ldg(M + (M_JINV + q) * v + gc);
          }
          const double rIp = Ac[A_Q0 * N2 + xp], rIm = Ac[A_Q0 * N2 + xm];
          const double rJp = Ac[A_Q0 * N2 + yp], rJm = Ac[A_Q0 * N2 + ym];
          const double rKp = Ap[A_Q0 * N2 + c2], rKm = Am[A_Q0 * N2 + c2];
          const double invI = Ac[A_RI * N2 + xp] * Ac[A_RI * N2 + xm];
          const double invJ = Ac[A_RI * N2 + yp] * Ac[A_RI * N2 + ym];
          const double invK = Ap[A_RI * N2 + c2] * Am[A_RI * N2 + c2];
#pragma unroll
          for (int l = 0; l < 4; l++) {
            double d0, d1, d2;
            if (l == 3) {
              d0 = 0.5 * (Ac[A_T * N2 + xp] - Ac[A_T * N2 + xm]);
              d1 = 0.5 * (Ac[A_T * N2 + yp] - Ac[A_T * N2 + ym]);
              d2 = 0.5 * (Ap[A_T * N2 + c2] - Am[A_T * N2 + c2]);
            } else {
              const int f = (A_Q1 + l) * N2;
              d0 = 0.5 * (Ac[f + xp] * rIm - Ac[f + xm] * rIp) * invI;
              d1 = 0.5 * (Ac[f + yp] * rJm - Ac[f + ym] * rJp) * invJ;
              d2 = 0.5 * (Ap[f + c2] * rKm - Am[f + c2] * rKp) * invK;
            }
#pragma unroll
            for (int e = 0; e < 3; e++) Gs[(3 * l + e) * N1 + r] = d0 * Jm[e] + d1 * Jm[3 + e] + d2 * Jm[6 + e];
          }
        }
      }
    };

    // the flux of one face of axis ax between R2 cells cL (plane pL) and cR (plane pR);
    // gL, gR are the R1 indices of the two cells (for the gradients)
    auto face = [&](int ax, const double *AL, int cL, const double *AR, int cR, const double *GL, int gL,
                    const double *GR, int gR, long long gcL, long long gcR, double *F) {
      KSide sl, sr;
      const double q0L = AL[A_Q0 * N2 + cL], q0R = AR[A_Q0 * N2 + cR];
      const double riL = AL[A_RI * N2 + cL], riR = AR[A_RI * N2 + cR];
      const double q1L = AL[A_Q1 * N2 + cL], q2L = AL[A_Q2 * N2 + cL], q3L = AL[A_Q3 * N2 + cL];
      const double q1R = AR[A_Q1 * N2 + cR], q2R = AR[A_Q2 * N2 + cR], q3R = AR[A_Q3 * N2 + cR];
      const double TL = AL[A_T * N2 + cL], TR = AR[A_T * N2 + cR];
      sl.u = quot(q1L, q0L, riL), sl.v = quot(q2L, q0L, riL), sl.w = quot(q3L, q0L, riL);
      sr.u = quot(q1R, q0R, riR), sr.v = quot(q2R, q0R, riR), sr.w = quot(q3R, q0R, riR);
      sl.p = q0L * kSp.R1 * TL, sr.p = q0R * kSp.R1 * TR;
      sl.rho = q0L, sr.rho = q0R;
      sl.e = AL[A_E * N2 + cL], sr.e = AR[A_E * N2 + cR];
      sl.th = kSp.th1 * TL, sr.th = kSp.th1 * TR;
      double S0, S1, S2;
      FaceGeom g;
      if constexpr (UNIFORM) {
        S0 = ax == 0 ? B.S[0] : 0.0;
        S1 = ax == 1 ? B.S[1] : 0.0;
        S2 = ax == 2 ? B.S[2] : 0.0;
        if constexpr (VISC) {
          g.S0 = S0, g.S1 = S1, g.S2 = S2;
          g.dampx = ax == 0 ? B.damp[0] : 0.0;
          g.dampy = ax == 1 ? B.damp[1] : 0.0;
          g.dampz = ax == 2 ? B.damp[2] : 0.0;
          g.xLx = ax == 0 ? B.xL[0] : 0.0, g.xLy = ax == 1 ? B.xL[1] : 0.0, g.xLz = ax == 2 ? B.xL[2] : 0.0;
          g.xRx = ax == 0 ? B.xR[0] : 0.0, g.xRy = ax == 1 ? B.xR[1] : 0.0, g.xRz = ax == 2 ? B.xR[2] : 0.0;
        }
      } else {
        S0 = __ldg(M + (M_S + 3 * ax) * v + gcR);
        S1 = __ldg(M + (M_S + 3 * ax + 1) * v + gcR);
        S2 = __ldg(M + (M_S + 3 * ax + 2) * v + gcR);
        if constexpr (VISC) {
          const double xf[3] = {__ldg(M + (M_XF + 3 * ax) * v + gcR), __ldg(M + (M_XF + 3 * ax + 1) * v + gcR),
                                __ldg(M + (M_XF + 3 * ax + 2) * v + gcR)};
          const double xl[3] = {__ldg(M + (M_XCC + 0) * v + gcL), __ldg(M + (M_XCC + 1) * v + gcL),
                                __ldg(M + (M_XCC + 2) * v + gcL)};
          const double xr[3] = {__ldg(M + (M_XCC + 0) * v + gcR), __ldg(M + (M_XCC + 1) * v + gcR),
                                __ldg(M + (M_XCC + 2) * v + gcR)};
          g = face_geom(S0, S1, S2, xf, xl, xr);
        }
      }
      double C;
      kepaec(sl, sr, S0, S1, S2, F, C);
      if constexpr (VISC) {
        double gl[12], gr[12];
#pragma unroll
        for (int q = 0; q < 12; q++) gl[q] = GL[q * N1 + gL], gr[q] = GR[q * N1 + gR];
        viscous1(g, kSp.mu1, kSp.kappa1, q1L * riL, q2L * riL, q3L * riL, TL, q1R * riR, q2R * riR, q3R * riR,
                 TR, gl, gr, F);
      }
    };

    // R2 / R1 index of a tile cell (ti, tj) and its global cell index at plane p
    auto c2of = [&](int ti, int tj) { return (ti + 2) + W2 * (tj + 2); };
    auto c1of = [&](int ti, int tj) { return (ti + 1) + W1 * (tj + 1); };
    auto gidx = [&](int ti, int tj, int p) {
      return (long long)(p + NG) * sK + (long long)(T.j0 + NG + tj) * sJ + (T.i0 + NG + ti);
    };

    const bool mine = tid < tw * th;
    const int ti = tid % tw, tj = tid / tw;
    double Fk[5];  // the k face below this thread's cell

    // the k face above plane p for this thread's cell
    auto kface = [&](int p, double *F) {
      const double *AL = A + slot3(p) * A_N * N2, *AR = A + slot3(p + 1) * A_N * N2;
      const double *GL = G + slot2(p) * 12 * N1, *GR = G + slot2(p + 1) * 12 * N1;
      face(2, AL, c2of(ti, tj), AR, c2of(ti, tj), GL, c1of(ti, tj), GR, c1of(ti, tj), gidx(ti, tj, p),
           gidx(ti, tj, p + 1), F);
    };

    // prelude: planes k0-2 .. k0+1 loaded, gradients of k0-1 and k0, the k face below k0
    const int k0 = T.k0, k1 = T.k1;
    load_plane(k0 - 2);
    load_plane(k0 - 1);
    load_plane(k0);
    __syncthreads();
    grad_plane(k0 - 1);
    __syncthreads();
    load_plane(k0 + 1);
    __syncthreads();
    grad_plane(k0);
    __syncthreads();
    if (mine) kface(k0 - 1, Fk);
    // the first load of the loop takes plane k0-1's slot, which that k face read
    __syncthreads();

    for (int k = k0; k < k1; k++) {
      load_plane(k + 2);
      __syncthreads();
      grad_plane(k + 1);
      __syncthreads();
      // the i and j faces of plane k
      {
        const double *Ac = A + slot3(k) * A_N * N2;
        const double *Gc = G + slot2(k) * 12 * N1;
        const int ni = (tw + 1) * th, nj = tw * (th + 1);
        for (int f = tid; f < ni + nj; f += FUSED_THREADS) {
          int ax, fi, fj;
          if (f < ni) {
            ax = 0, fi = f % (tw + 1), fj = f / (tw + 1);
          } else {
            ax = 1, fi = (f - ni) % tw, fj = (f - ni) / tw;
          }
          // the face's right cell is tile cell (fi, fj); its left one step back along ax
          const int cR = c2of(fi, fj), cL = cR - (ax == 0 ? 1 : W2);
          const int gR = c1of(fi, fj), gL = gR - (ax == 0 ? 1 : W1);
          const long long gcR = gidx(fi, fj, k), gcL = gcR - (ax == 0 ? 1 : sJ);
          double F[5];
          face(ax, Ac, cL, Ac, cR, Gc, gL, Gc, gR, gcL, gcR, F);
          double *Fs = ax == 0 ? Fi : Fj;
#pragma unroll
          for (int l = 0; l < 5; l++) Fs[l * N1 + gR] = F[l];
        }
      }
      double Fkh[5];
      if (mine) kface(k, Fkh);
      __syncthreads();
      if (mine) {
        const int g1 = c1of(ti, tj);
        const long long gc = gidx(ti, tj, k);
        const double dJ = UNIFORM ? B.detJinv : __ldg(M + M_DETJINV * v + gc);
        double dQ[5];
#pragma unroll
        for (int l = 0; l < 5; l++)
          dQ[l] = (Fi[l * N1 + g1] + Fj[l * N1 + g1] + Fk[l] - Fi[l * N1 + g1 + 1] - Fj[l * N1 + g1 + W1] - Fkh[l]) * dJ;
        const double dt = *a.dt;
        const long long base = 5 * B.cv + gc;
        double first[5];
#pragma unroll
        for (int m = 0; m < 2; m++) {
          if (m >= a.ncomb) break;
          const FusedCombine &cb = a.comb[m];
          double *out = a.R[cb.out] + base;
#pragma unroll
          for (int l = 0; l < 5; l++) {
            auto val = [&](int n) {
              const int s = cb.src[n];
              return s == -1 ? dQ[l] : s == -2 ? first[l] : a.R[s][base + l * v];
            };
            auto term = [&](int n) { return (cb.step && n == cb.nterms - 1) ? cb.w[n] * dt * val(n) : cb.w[n] * val(n); };
            double acc = term(0);
#pragma unroll
            for (int n = 1; n < 4; n++)
              if (n < cb.nterms) acc = acc + term(n);
            if (m == 0) first[l] = acc;
            if (cb.write) out[l * v] = acc;
          }
        }
#pragma unroll
        for (int l = 0; l < 5; l++) Fk[l] = Fkh[l];
      }
    }
    __syncthreads();
  }
}

// the shared memory a tile of tw x th takes
inline size_t fused_smem(int tw, int th, bool visc) {
  const int N2 = (tw + 4) * (th + 4), N1 = (tw + 2) * (th + 2);
  return sizeof(double) * (size_t)(3 * A_N * N2 + (visc ? 2 * 12 * N1 : 0) + 10 * N1);
}

}  // namespace pgb
