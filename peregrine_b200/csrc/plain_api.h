// The per-block path's entry points, one set per species count: each is
// compiled from plain_tu.cu with PGB_NS set, so a species count's kernels
// build in their own translation unit (and in parallel).  Internal to the
// library (hidden visibility); the C ABI is include/pgb200.h.
#pragma once
#include <cuda_runtime.h>

#include "bc_types.h"
#include "chem_types.h"
#include "layout.cuh"
#include "physics.cuh"

namespace pgb {

// the ranges a pass runs over
enum { R_VOL = 0, R_INNER = 1, R_FX = 2, R_FY = 3, R_FZ = 4 };
inline long long range_size(const BlockDev &D, int r) {
  switch (r) {
    case R_VOL: return D.vol;
    case R_INNER: return (long long)D.nx * D.ny * D.nz;
    case R_FX: return (long long)(D.nx + 1) * D.ny * D.nz;
    case R_FY: return (long long)D.nx * (D.ny + 1) * D.nz;
    default: return (long long)D.nx * D.ny * (D.nz + 1);
  }
}

// what a right-hand side on the per-block path reads of a case
struct PlainCase {
  const BlockDev *d_blks;  // device descriptors
  const BlockDev *h_blks;  // the same on the host, for the launch sizes
  int nblocks;
  double *state, *tr, *hsp, *grads, *F[3];
  const double *met;
  const HaloEntry *halo;
  long long nhalo, nhalo_l0;  // every halo entry; the first layer's
  // the same halo as boxes (k_halo_boxes), when the case has them: the
  // boxes, the CTA table, its length, the cells no box holds
  const HaloPatch *boxes;
  const int2 *boxcta;
  long long nboxcta;
  const HaloEntry *boxrest;
  long long nboxrest;
  // the first face layer alone as boxes (the gradients' fill), when the case
  // lists its halo only as boxes
  const HaloPatch *boxes0;
  const int2 *boxcta0;
  long long nboxcta0;
  const double *rots;         // the rotationally periodic interfaces' rotations, 3 x 3 each
  int visc, primary, recon, limiter;
  int chem;  // 0 none, 1 coupled source, 2 sub-stepped (PGB_CHEM_*)
  // the sub-stepped chemistry: its options, each cell's last substep count
  // (every block's full layout, end to end) and the stiff list
  SubstepOpts subopt;
  int *subs;
  StiffList stiff;
  int realgas;  // the cubic real gas: the kernels built for it
  int df;      // the double flux: fromplane in the stages, two energy rows per face (F holds NE + 1 rows)
  int packed;  // 1: each pass is one launch over every block
  // with packing, each range's tile table (cells with halo, interior cells,
  // i, j and k faces): CTA x works tile ctab[r][x].y of block ctab[r][x].x;
  // without a table a packed launch gives each block a grid row
  const int2 *ctab[5];
  long long nctab[5];
  // boundaries: the face tables of the halo, gradient and wall passes (each
  // ending in its sentinel) and their face counts, the entries, their value
  // programs, the clock and dt in device memory and the stage's time as a
  // fraction of dt
  const BcFace *bchalo, *bcgrad, *bcwall;
  int nbchalo, nbcgrad, nbcwall;
  long long bchalo_n, bcgrad_n, bcwall_n;
  const BcEntry *bcent;
  const BcOp *bcops;
  const double *clock, *dt;
  // the coupled source generated for the mechanism (a kernel handle for
  // cudaLaunchKernel; null for the table-driven kernel), the table log's and
  // exp's tables it reads, and the block record's size
  const void *gensrc, *genmath;
  int blkstride;
  // the fused passes' cell pass over the interior cells, its fields then
  // copied into the halo (blocks whose halo is a large share of their cells)
  int rcell_inner;
  double tfrac;
  cudaStream_t stream;
  void (*mark)(void *ctx, int kind);  // called after each launch, kind 0 halo, 2 block, 4 boundary, 5 CFL
  void *ctx;
};

// The fused passes' stage (react.cuh): the stage's register, dQ (the
// coupled source's home and, with write_dq, dQ's), and the combines on
// physical registers: out = sum_n w[n] X[n] left to right, dt on the last
// term when step is set, a term's src -1 for dQ and -2 for the first
// combine's value at the cell; write 0 drops a store no later stage reads.
struct RCombine {
  double *out;
  const double *X[4];
  double w[4];
  int src[4];
  int nterms, step, write;
};
struct RStage {
  const double *Q;
  double *dQ;
  int write_dq;
  int ncomb;
  RCombine comb[2];
};

// the serving pool's reactors' stage (react.cuh, k_reactors): the stage's
// register and each reactor's last T, the running rows, the table's
// capacity, the step size and the stage's combines on the reactor registers
struct ReactorStage {
  const double *Q;
  double *T;
  const int *rows;
  int n;
  long long cap;
  const double *dt;
  int ncomb;
  RCombine comb[2];
};

struct PlainOps {
  int (*upload)(const Species *, const Mech *, const MathTables *, cudaStream_t);
  int (*rhs)(const PlainCase *, const double *Q, double *dQ);
  int (*fromprims)(const PlainCase *, int blk, const double *prims, double *Q);
  int (*production)(long long n, const double *rho, const double *Y, const double *T, double *omega, cudaStream_t);
  int (*prestep)(const PlainCase *, double *Q, int first);
  int (*cflmax)(const PlainCase *, const double *Q, double *out);
  int (*fused)(const PlainCase *, const RStage *);
  int (*reactors)(const ReactorStage *, cudaStream_t);
  int (*reactor_prims)(const double *prims, double *Q, double *T, int row, long long cap, cudaStream_t);
};

}  // namespace pgb

#define PGB_PLAIN_DECL(N) PGB_PLAIN_DECL_I(N)
#define PGB_PLAIN_DECL_I(N)                                                                                      \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_upload_##N(                                     \
      const pgb::Species *, const pgb::Mech *, const pgb::MathTables *, cudaStream_t);                           \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_rhs_##N(const pgb::PlainCase *, const double *, \
                                                                         double *);                              \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_fromprims_##N(const pgb::PlainCase *, int,      \
                                                                               const double *, double *);        \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_production_##N(                                 \
      long long, const double *, const double *, const double *, double *, cudaStream_t);                        \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_prestep_##N(const pgb::PlainCase *, double *, int); \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_cflmax_##N(const pgb::PlainCase *, const double *,  \
                                                                            double *);                           \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_fused_##N(const pgb::PlainCase *,               \
                                                                           const pgb::RStage *);                 \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_reactors_##N(const pgb::ReactorStage *,         \
                                                                              cudaStream_t);                     \
  extern "C" __attribute__((visibility("hidden"))) int pgb_plain_reactor_prims_##N(                              \
      const double *, double *, double *, int, long long, cudaStream_t);
