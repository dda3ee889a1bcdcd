// The per-block path for one species count, PGB_NS (1 when unset): the
// reference's passes one by one, one launch per block and kernel, each pass a
// round trip through HBM as in the reference's rhs graph
// (peregrine/simulator/advec/simulator.py:57-87,
// peregrine/simulator/advecdiff/simulator.py:110-124), with the coupled
// chemistry source beginning dQ (peregrine/simulator/chemint/coupled.py).
// The build compiles this file once per species count.
#include <algorithm>
#include <string>

#include "bc.cuh"
#include "cfl.cuh"
#include "chem.cuh"
#include "pgb200.h"
#include "substep.cuh"
#include "plain.cuh"
#include "plain_api.h"
#include "react.cuh"

#ifndef PGB_NS
#define PGB_NS 1
#endif

extern "C" __attribute__((visibility("hidden"))) int pgb_internal_fail(int code, const char *msg);

namespace pgb {
namespace {

constexpr int NS = PGB_NS;
constexpr int NE = 4 + NS;
constexpr int TH = 256;

unsigned grid_of(long long n) { return (unsigned)std::max<long long>(1, (n + TH - 1) / TH); }

// the sub-stepped chemistry's stiff pass: its persistent grid, every SM
// filled with its CTAs (set when the unit's tables are uploaded, outside any
// stream capture)
int g_stiff_ctas = 148;

int cuda_fail(cudaError_t e, const char *what) {
  return pgb_internal_fail(e == cudaErrorMemoryAllocation ? PGB_ERR_NOMEM : PGB_ERR_CUDA,
                           (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

void mark(const PlainCase *pc, int kind) {
  if (pc->mark) pc->mark(pc->ctx, kind);
}

// the full halo of a register (comps components, vec the component its
// rotations turn): by boxes when the case has them, else by entries
// the gradients' fill: the first face layer, each row's directions and the
// velocity rows turned across a rotational periodic
void grads_fill(const PlainCase *pc) {
  constexpr int NG3 = 3 * (NE - 1);
  if (pc->boxcta0 && pc->nboxcta0 > 0)
    halo_boxes_launch<NG3>((unsigned)pc->nboxcta0, pc->stream, pc->grads, pc->boxes0, pc->boxcta0, nullptr, 0, NG3,
                           HALO_TENSOR, pc->rots);
  else
    k_halo<<<grid_of(pc->nhalo_l0), TH, 0, pc->stream>>>(pc->grads, pc->halo, pc->nhalo_l0, NG3, HALO_TENSOR,
                                                        pc->rots);
}

void halo_fill(const PlainCase *pc, double *base, int comps, int vec, int stride = 0) {
  if (pc->boxcta && pc->nboxcta > 0)
    halo_boxes_launch<NE, SW>((unsigned)pc->nboxcta, pc->stream, base, pc->boxes, pc->boxcta, pc->boxrest, pc->nboxrest,
                              comps, vec, pc->rots, stride);
  else
    k_halo<<<grid_of(pc->nhalo), TH, 0, pc->stream>>>(base, pc->halo, pc->nhalo, comps, vec, pc->rots, stride);
}

// a pass over every block: one launch per block, or packed, one launch over
// them all, by the range's tile table when there is one, else a grid row per
// block as long as the largest block needs
typedef void (*Launch)(const PlainCase *, int, dim3, const int2 *, const void *);

void for_blocks(const PlainCase *pc, int range, Launch launch, const void *ctx, int kind) {
  if (pc->packed) {
    if (pc->ctab[range]) {
      if (pc->nctab[range] > 0) launch(pc, 0, dim3((unsigned)pc->nctab[range], 1, 1), pc->ctab[range], ctx);
    } else {
      long long most = 0;
      for (int b = 0; b < pc->nblocks; b++) most = std::max(most, range_size(pc->h_blks[b], range));
      if (pc->nblocks > 0) launch(pc, 0, dim3(grid_of(most), (unsigned)pc->nblocks, 1), nullptr, ctx);
    }
    mark(pc, kind);
  } else {
    for (int b = 0; b < pc->nblocks; b++) {
      launch(pc, b, dim3(grid_of(range_size(pc->h_blks[b], range)), 1, 1), nullptr, ctx);
      mark(pc, kind);
    }
  }
}

struct RhsArgs {
  const double *Q;
  double *dQ;
};

template <int A, bool RG>
void riemann_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const RhsArgs &a, int lim) {
  cudaStream_t s = pc->stream;
  switch (pc->primary) {
    case PGB_FLUX_HLLC: k_riemann<NS, A, FN_HLLC, RG><<<g, TH, 0, s>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->F[A], lim, ct); break;
    case PGB_FLUX_RUSANOV: k_riemann<NS, A, FN_RUSANOV, RG><<<g, TH, 0, s>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->F[A], lim, ct); break;
    default: k_riemann<NS, A, FN_AUSMUP, RG><<<g, TH, 0, s>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->F[A], lim, ct); break;
  }
}

// the double flux's Riemann forms (Rusanov, AUSM+-up; the case refuses HLLC)
template <int A>
void riemann_df_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const RhsArgs &a, int lim) {
  cudaStream_t s = pc->stream;
  if (pc->primary == PGB_FLUX_RUSANOV)
    k_riemann<NS, A, FN_RUSANOV, true, true><<<g, TH, 0, s>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->F[A], lim, ct);
  else
    k_riemann<NS, A, FN_AUSMUP, true, true><<<g, TH, 0, s>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->F[A], lim, ct);
}

template <int A>
void adv_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  const int lim = pc->recon == PGB_RECON_MUSCL ? pc->limiter : 0;
  cudaStream_t s = pc->stream;
  if (pc->df) {
    if (pc->primary == PGB_FLUX_KEPAEC)
      k_advflux_df<NS, A><<<g, TH, 0, s>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->F[A], ct);
    else
      riemann_df_launch<A>(pc, b, g, ct, a, lim);
    return;
  }
  if (pc->primary == PGB_FLUX_KEPAEC) {
    k_advflux<NS, A><<<g, TH, 0, s>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->F[A], ct);
  } else if (pc->realgas) {
    riemann_launch<A, true>(pc, b, g, ct, a, lim);
  } else {
    riemann_launch<A, false>(pc, b, g, ct, a, lim);
  }
}

template <int A>
void diff_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  if (pc->df)
    k_diffflux<NS, A, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, pc->tr, pc->hsp, pc->grads, pc->met, pc->F[A], ct);
  else
    k_diffflux<NS, A><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, pc->tr, pc->hsp, pc->grads, pc->met, pc->F[A], ct);
}

// the double flux's state off the frozen planes on the interior alone (R_INNER)
void fromplane_inner_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  k_fromQ<NS, true, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, ct, 1);
}
void fromQ_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  if (pc->realgas)
    k_fromQ<NS, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, ct, pc->df);
  else
    k_fromQ<NS, false><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, ct, 0);
}
void transport_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  if (pc->realgas)
    k_transport<NS, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, pc->tr, pc->hsp, ct);
  else
    k_transport<NS, false><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, pc->tr, pc->hsp, ct);
}
void grads_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  k_grads<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, pc->met, pc->grads, 0, ct);
}
// the coupled source: the kernel generated for the case's mechanism where it
// has one (rategen.cu), else the table-driven k_source
void launch_source(const PlainCase *pc, int b, dim3 g, const int2 *ct, const double *Q, double *dQ) {
  if (pc->gensrc) {
    const char *blks = reinterpret_cast<const char *>(pc->d_blks);
    int stride = pc->blkstride, blk = b;
    const double *st = pc->state;
    const void *mt = pc->genmath;
    void *args[] = {&blks, &stride, &blk, &Q, &st, &dQ, &ct, &mt};
    cudaLaunchKernel(pc->gensrc, g, dim3(TH), args, 0, pc->stream);
    return;
  }
  k_source<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, Q, pc->state, dQ, ct);
}
void source_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  launch_source(pc, b, g, ct, a.Q, a.dQ);
}
void bulk_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  k_substep_bulk<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, a.dQ, pc->subs, pc->dt, pc->subopt,
                                               pc->stiff, ct);
}
void apply_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RhsArgs &a = *(const RhsArgs *)ctx;
  if (pc->df)
    k_applyflux_df<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, pc->F[0], pc->F[1], pc->F[2], pc->met, a.dQ, ct);
  else
    k_applyflux<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, pc->F[0], pc->F[1], pc->F[2], pc->met, a.dQ, pc->chem, ct);
}

}  // namespace
}  // namespace pgb

using namespace pgb;

#define PGB_CAT2(a, b) a##b
#define PGB_CAT(a, b) PGB_CAT2(a, b)
#define PGB_ENTRY(name) PGB_CAT(name, PGB_NS)

PGB_PLAIN_DECL(PGB_NS)

// the species, mechanism and math tables into this unit's constant and
// global memory
extern "C" int PGB_ENTRY(pgb_plain_upload_)(const Species *sp, const Mech *mech, const MathTables *mt,
                                            cudaStream_t s) {
  cudaError_t e = cudaMemcpyToSymbolAsync(kSp, sp, sizeof(Species), 0, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "species constants");
  if (mech) {
    e = cudaMemcpyToSymbolAsync(kMech, mech, sizeof(Mech), 0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "mechanism constants");
    e = cudaMemcpyToSymbolAsync(gMech, mech, sizeof(Mech), 0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "mechanism tables");
  }
  if (mt) {
    e = cudaMemcpyToSymbolAsync(gMath, mt, sizeof(MathTables), 0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "math tables");
    int per_sm = 0, sms = 148, dev = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_substep_stiff<NS>, 128, 0) != cudaSuccess) per_sm = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    g_stiff_ctas = sms * std::max(1, per_sm);
  }
  return PGB_OK;
}

// the boundary passes: the halo cells behind every boundary face (after the
// state, before the transport reads them), the inflows' and outflows' halo
// gradients (after the gradients' exchange) and the walls' face fluxes (after
// the flux functions, before the divergence), one launch each over every
// block's boundary faces
static void bc_halo_launch(const PlainCase *pc, const double *Q) {
  if (!pc->nbchalo) return;
  if (pc->realgas)
    k_bc_halo<NS, true><<<grid_of(pc->bchalo_n), TH, 0, pc->stream>>>(
        pc->d_blks, pc->bchalo, pc->nbchalo, pc->bcent, pc->bcops, const_cast<double *>(Q), pc->state, pc->met,
        pc->clock, pc->dt, pc->tfrac);
  else
    k_bc_halo<NS, false><<<grid_of(pc->bchalo_n), TH, 0, pc->stream>>>(
        pc->d_blks, pc->bchalo, pc->nbchalo, pc->bcent, pc->bcops, const_cast<double *>(Q), pc->state, pc->met,
        pc->clock, pc->dt, pc->tfrac);
  mark(pc, 4);
}
static void bc_grads_launch(const PlainCase *pc) {
  if (!pc->nbcgrad) return;
  k_bc_grads<NS><<<grid_of(pc->bcgrad_n), TH, 0, pc->stream>>>(pc->d_blks, pc->bcgrad, pc->nbcgrad, pc->grads);
  mark(pc, 4);
}
static void bc_wall_launch(const PlainCase *pc, const double *Q) {
  if (!pc->nbcwall) return;
  k_bc_wall<NS><<<grid_of(pc->bcwall_n), TH, 0, pc->stream>>>(
      pc->d_blks, pc->bcwall, pc->nbcwall, pc->bcent, pc->bcops, Q, pc->state, pc->tr, pc->met, pc->F[0], pc->F[1],
      pc->F[2], NE + (pc->df ? 1 : 0), pc->visc, pc->clock, pc->dt, pc->tfrac);
  mark(pc, 4);
}

// the sub-stepped chemistry's passes: the list's header cleared, the bulk
// pass over every block (it lists the cells short of the step's end), and,
// compacted, the stiff pass over the list, one persistent launch
static void substep_passes(const PlainCase *pc, const RhsArgs &a) {
  const SubstepOpts &o = pc->subopt;
  cudaMemsetAsync(pc->stiff.head, 0, sizeof(unsigned int) * (o.bins + 2), pc->stream);
  for_blocks(pc, R_INNER, bulk_launch, &a, 6);
  if (o.bulk < o.cap) {
    k_substep_stiff<NS><<<g_stiff_ctas, 128, 0, pc->stream>>>(pc->d_blks, a.Q, pc->state, a.dQ, pc->subs, pc->dt,
                                                               o, pc->stiff);
    mark(pc, 7);
  }
}

// one right-hand side of every block: Q's halo, the state everywhere, the
// boundaries' halo cells, the transport and gradients on the viscous path
// (the gradients' first halo layer exchanged or set by the boundaries), the
// chemistry source, the face fluxes per axis, the walls' fluxes and the
// divergence (peregrine/simulator/advec/simulator.py:57-84,
// peregrine/simulator/advecdiff/simulator.py:110-124).  Per block the passes
// run block by block (the reference's order); packed, each pass is one launch
// over every block.
extern "C" int PGB_ENTRY(pgb_plain_rhs_)(const PlainCase *pc, const double *Q, double *dQ) {
  cudaStream_t s = pc->stream;
  const RhsArgs a{Q, dQ};
  halo_fill(pc, const_cast<double *>(Q), NE, 1);
  mark(pc, 0);
  if (pc->packed) {
    for_blocks(pc, R_VOL, fromQ_launch, &a, 2);
    bc_halo_launch(pc, Q);
    if (pc->visc) {
      for_blocks(pc, R_VOL, transport_launch, &a, 2);
      for_blocks(pc, R_INNER, grads_launch, &a, 2);
    }
  } else {
    for (int b = 0; b < pc->nblocks; b++) {
      fromQ_launch(pc, b, dim3(grid_of(pc->h_blks[b].vol)), nullptr, &a);
      mark(pc, 2);
    }
    bc_halo_launch(pc, Q);
    if (pc->visc) {
      for (int b = 0; b < pc->nblocks; b++) {
        const BlockDev &D = pc->h_blks[b];
        transport_launch(pc, b, dim3(grid_of(D.vol)), nullptr, &a);
        mark(pc, 2);
        grads_launch(pc, b, dim3(grid_of(range_size(D, R_INNER))), nullptr, &a);
        mark(pc, 2);
      }
    }
  }
  if (pc->visc) {
    grads_fill(pc);
    mark(pc, 0);
    bc_grads_launch(pc);
  }
  if (pc->chem == PGB_CHEM_SUBSTEPPED) substep_passes(pc, a);
  if (pc->packed) {
    if (pc->chem == PGB_CHEM_COUPLED) for_blocks(pc, R_INNER, source_launch, &a, 2);
    for_blocks(pc, R_FX, adv_launch<0>, &a, 2);
    for_blocks(pc, R_FY, adv_launch<1>, &a, 2);
    for_blocks(pc, R_FZ, adv_launch<2>, &a, 2);
    if (pc->visc) {
      for_blocks(pc, R_FX, diff_launch<0>, &a, 2);
      for_blocks(pc, R_FY, diff_launch<1>, &a, 2);
      for_blocks(pc, R_FZ, diff_launch<2>, &a, 2);
    }
    bc_wall_launch(pc, Q);
    for_blocks(pc, R_INNER, apply_launch, &a, 2);
  } else {
    for (int b = 0; b < pc->nblocks; b++) {
      const BlockDev &D = pc->h_blks[b];
      auto g = [&](int r) { return dim3(grid_of(range_size(D, r))); };
      if (pc->chem == PGB_CHEM_COUPLED) {
        source_launch(pc, b, g(R_INNER), nullptr, &a);
        mark(pc, 2);
      }
      adv_launch<0>(pc, b, g(R_FX), nullptr, &a);
      mark(pc, 2);
      adv_launch<1>(pc, b, g(R_FY), nullptr, &a);
      mark(pc, 2);
      adv_launch<2>(pc, b, g(R_FZ), nullptr, &a);
      mark(pc, 2);
      if (pc->visc) {
        diff_launch<0>(pc, b, g(R_FX), nullptr, &a);
        mark(pc, 2);
        diff_launch<1>(pc, b, g(R_FY), nullptr, &a);
        mark(pc, 2);
        diff_launch<2>(pc, b, g(R_FZ), nullptr, &a);
        mark(pc, 2);
      }
      // without walls a block's divergence follows its own fluxes
      if (!pc->nbcwall) {
        apply_launch(pc, b, g(R_INNER), nullptr, &a);
        mark(pc, 2);
      }
    }
    if (pc->nbcwall) {
      bc_wall_launch(pc, Q);
      for (int b = 0; b < pc->nblocks; b++) {
        apply_launch(pc, b, dim3(grid_of(range_size(pc->h_blks[b], R_INNER))), nullptr, &a);
        mark(pc, 2);
      }
    }
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "per-block launch");
}

// the CFL reduction of register Q over every block's interior into out[0..2],
// which the caller zeroed: one launch, a grid row per block
extern "C" int PGB_ENTRY(pgb_plain_cflmax_)(const PlainCase *pc, const double *Q, double *out) {
  long long most = 0;
  for (int b = 0; b < pc->nblocks; b++) {
    const BlockDev &D = pc->h_blks[b];
    most = std::max(most, (long long)D.nx * D.ny * D.nz);
  }
  // about eight CTAs per SM in all, each striding over its block's cells
  const long long want = std::max<long long>(1, (8 * 148 + pc->nblocks - 1) / pc->nblocks);
  const dim3 g((unsigned)std::min<long long>(grid_of(most), want), (unsigned)pc->nblocks, 1);
  if (pc->realgas)
    k_cflmax<NS, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, 0, Q, pc->state, pc->met, out, pc->df);
  else
    k_cflmax<NS, false><<<g, TH, 0, pc->stream>>>(pc->d_blks, 0, Q, pc->state, pc->met, out, 0);
  mark(pc, 5);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "cflmax");
}

// Q and the state of one block's interior from its primitives
extern "C" int PGB_ENTRY(pgb_plain_fromprims_)(const PlainCase *pc, int blk, const double *prims, double *Q) {
  const BlockDev &D = pc->h_blks[blk];
  if (pc->realgas)
    k_fromprims<NS, true><<<grid_of((long long)D.nx * D.ny * D.nz), TH, 0, pc->stream>>>(pc->d_blks, blk, prims, Q, pc->state);
  else
    k_fromprims<NS, false><<<grid_of((long long)D.nx * D.ny * D.nz), TH, 0, pc->stream>>>(pc->d_blks, blk, prims, Q, pc->state);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "fromprims");
}

// the fold alone on independent states (device arrays)
extern "C" int PGB_ENTRY(pgb_plain_production_)(long long n, const double *rho, const double *Y, const double *T,
                                                double *omega, cudaStream_t s) {
  if (n > 0) k_production<NS><<<grid_of(n), TH, 0, s>>>(n, rho, Y, T, omega);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "production");
}

namespace {
struct PrestepArgs {
  double *Q;
  int first;
};
void prestep_fromQ_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const PrestepArgs &a = *(const PrestepArgs *)ctx;
  k_fromQ<NS, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, ct, a.first ? 0 : 1);
}
void prestep_fromQ_inner_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const PrestepArgs &a = *(const PrestepArgs *)ctx;
  k_fromQ<NS, true, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, ct, a.first ? 0 : 1);
}
void prestep_freeze_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const PrestepArgs &a = *(const PrestepArgs *)ctx;
  k_freeze<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, a.Q, pc->state, ct);
}
}  // namespace

// the double flux's step start: the state of Q (the eos's fromrhoE on the
// first step, the frozen planes' after), the planes frozen anew on the
// interior with the energy reset to the eos's, then Q and the state (planes
// included) copied into the halos, so a halo's plane is its image's (one
// pass for both where the halo goes by boxes)
// (peregrine/simulator/eulerdf/simulator.py:58-66)
extern "C" int PGB_ENTRY(pgb_plain_prestep_)(const PlainCase *pc, double *Q, int first) {
  cudaStream_t s = pc->stream;
  if (pc->packed) {
    // each pass one launch over every block
    const PrestepArgs pa{Q, first};
    // the halo's state is the copy below, so with rcell_inner only the
    // interior's is formed (a boundary's halo cells keep the whole pass)
    if (pc->rcell_inner && !pc->nbchalo)
      for_blocks(pc, R_INNER, prestep_fromQ_inner_launch, &pa, 2);
    else
      for_blocks(pc, R_VOL, prestep_fromQ_launch, &pa, 2);
    for_blocks(pc, R_INNER, prestep_freeze_launch, &pa, 2);
  } else {
    for (int b = 0; b < pc->nblocks; b++) {
      const BlockDev &D = pc->h_blks[b];
      k_fromQ<NS, true><<<grid_of(D.vol), TH, 0, s>>>(pc->d_blks, b, Q, pc->state, nullptr, first ? 0 : 1);
      mark(pc, 2);
      k_freeze<NS><<<grid_of(range_size(D, R_INNER)), TH, 0, s>>>(pc->d_blks, b, Q, pc->state);
      mark(pc, 2);
    }
  }
  // the state's record up to its last plane field (p .. c, Z, theta, eps,
  // kappa and the NS - 1 zetas), the rest of its stride unused here
  constexpr int CS = ST_ZETA + NS - 1;
  if (pc->boxcta && pc->nboxcta > 0) {
    // Q's halo and the state's (planes included) in one pass over the boxes
    if (pc->rots)
      k_halo_boxes2<NE, CS, true><<<(unsigned)pc->nboxcta, 256, 0, s>>>(Q, 1, 0, pc->state, SW, pc->boxes, pc->boxcta,
                                                                        pc->boxrest, pc->nboxrest, pc->rots);
    else
      k_halo_boxes2<NE, CS, false><<<(unsigned)pc->nboxcta, 256, 0, s>>>(Q, 1, 0, pc->state, SW, pc->boxes, pc->boxcta,
                                                                         pc->boxrest, pc->nboxrest, pc->rots);
    mark(pc, 0);
  } else {
    halo_fill(pc, Q, NE, 1);
    mark(pc, 0);
    halo_fill(pc, pc->state, CS, HALO_SCALARS, SW);
    mark(pc, 0);
  }
  // the boundaries' halo cells from the state just formed, then their planes
  if (pc->nbchalo) {
    bc_halo_launch(pc, Q);
    k_bc_freeze<NS><<<grid_of(pc->bchalo_n), TH, 0, s>>>(pc->d_blks, pc->bchalo, pc->nbchalo, Q, pc->state);
    mark(pc, 4);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "double-flux freeze");
}

// The fused passes' stage (react.cuh): Q's halo, the cell pass (fromQ, the
// transport and the coupled source), the gradients and their first halo
// layer, and the tile kernel (every face, the divergence and the combines),
// each pass one launch over every block
namespace {
template <bool VISC>
void rcell_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RStage &r = *(const RStage *)ctx;
  k_rcell<NS, VISC><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, r.Q, pc->state, pc->tr, pc->hsp, ct);
}
template <bool VISC>
void rcell_inner_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RStage &r = *(const RStage *)ctx;
  k_rcell<NS, VISC, true><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, r.Q, pc->state, pc->tr, pc->hsp, ct);
}
void rsource_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RStage &r = *(const RStage *)ctx;
  launch_source(pc, b, g, ct, r.Q, r.dQ);
}
void rgrads_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RStage &r = *(const RStage *)ctx;
  k_grads<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, r.Q, pc->state, pc->met, pc->grads, 0, ct);
}
}  // namespace

namespace {
template <int A>
void rface_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RStage &r = *(const RStage *)ctx;
  const int lim = pc->recon == PGB_RECON_MUSCL ? pc->limiter : 0;
  cudaStream_t s = pc->stream;
#define PGB_RFACE(FN)                                                                                          \
  if (pc->visc)                                                                                              \
    k_rface<NS, A, FN, true><<<g, TH, 0, s>>>(pc->d_blks, b, r.Q, pc->state, pc->tr, pc->hsp, pc->grads,     \
                                              pc->met, pc->F[A], lim, ct);                                   \
  else                                                                                                       \
    k_rface<NS, A, FN, false><<<g, TH, 0, s>>>(pc->d_blks, b, r.Q, pc->state, pc->tr, pc->hsp, pc->grads,    \
                                               pc->met, pc->F[A], lim, ct);
  switch (pc->primary) {
    case PGB_FLUX_KEPAEC: PGB_RFACE(0) break;
    case PGB_FLUX_HLLC: PGB_RFACE(FN_HLLC) break;
    case PGB_FLUX_RUSANOV: PGB_RFACE(FN_RUSANOV) break;
    default: PGB_RFACE(FN_AUSMUP) break;
  }
#undef PGB_RFACE
}
struct RApplyCtx {
  RApplyArgs a;
};
void rapply_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RApplyCtx &r = *(const RApplyCtx *)ctx;
  k_rapply<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, pc->F[0], pc->F[1], pc->F[2], pc->met, r.a, ct);
}
struct RCellFluxCtx {
  const double *Q;
  RApplyArgs a;
};
void rcellflux_df_launch(const PlainCase *pc, int b, dim3 g, const int2 *ct, const void *ctx) {
  const RCellFluxCtx &r = *(const RCellFluxCtx *)ctx;
  k_rcellflux_df<NS><<<g, TH, 0, pc->stream>>>(pc->d_blks, b, r.Q, pc->state, pc->met, r.a, ct);
}
}  // namespace

extern "C" int PGB_ENTRY(pgb_plain_fused_)(const PlainCase *pc, const RStage *rs) {
  cudaStream_t s = pc->stream;
  // the double flux's interior state pass reads no halo cell: its stage
  // fills Q's halo after that pass, in the state's copy
  const bool df_inner = pc->df && pc->rcell_inner && pc->boxcta && pc->nboxcta > 0;
  if (!df_inner) {
    halo_fill(pc, const_cast<double *>(rs->Q), NE, 1);
    mark(pc, 0);
  }
  if (pc->df) {
    // the double flux, inviscid, kepaec: the state off each cell's frozen
    // plane (halo included), then a cell a thread of its six faces, the
    // divergence and the combines
    const RhsArgs q{rs->Q, rs->dQ};
    if (df_inner) {
      // the interior's state, then in one pass over the halo Q's halo and
      // each halo cell's state (p .. c and Z) copied from its source's: the
      // values the pass would form there, as a halo cell's Q, frozen plane
      // and last T are its source's
      for_blocks(pc, R_INNER, fromplane_inner_launch, &q, 8);
      constexpr int CS = ST_Z + 1;
      if (pc->rots)
        k_halo_boxes2<NE, CS, true><<<(unsigned)pc->nboxcta, 256, 0, s>>>(
            const_cast<double *>(rs->Q), 1, 0, pc->state, SW, pc->boxes, pc->boxcta, pc->boxrest, pc->nboxrest, pc->rots);
      else
        k_halo_boxes2<NE, CS, false><<<(unsigned)pc->nboxcta, 256, 0, s>>>(
            const_cast<double *>(rs->Q), 1, 0, pc->state, SW, pc->boxes, pc->boxcta, pc->boxrest, pc->nboxrest, pc->rots);
      mark(pc, 0);
    } else {
      for_blocks(pc, R_VOL, fromQ_launch, &q, 8);
    }
    RCellFluxCtx cf{};
    cf.Q = rs->Q;
    RApplyArgs &a = cf.a;
    a.dQ = rs->dQ;
    a.dt = pc->dt;
    a.write_dq = rs->write_dq;
    a.ncomb = rs->ncomb;
    a.comb[0] = rs->comb[0];
    a.comb[1] = rs->comb[1];
    for_blocks(pc, R_INNER, rcellflux_df_launch, &cf, 1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PGB_OK : cuda_fail(e, "fused double-flux stage");
  }
  if (pc->rcell_inner) {
    // the interior cells, then each halo cell's fields from its source's:
    // the same values, as a halo cell's Q and last T are its source's
    for_blocks(pc, R_INNER, pc->visc ? rcell_inner_launch<true> : rcell_inner_launch<false>, rs, 8);
    halo_fill(pc, pc->state, 8, HALO_SCALARS, SW);
    mark(pc, 0);
    if (pc->visc) {
      halo_fill(pc, pc->tr, 2 + NS, HALO_SCALARS);
      mark(pc, 0);
      halo_fill(pc, pc->hsp, NS, HALO_SCALARS);
      mark(pc, 0);
    }
  } else {
    for_blocks(pc, R_VOL, pc->visc ? rcell_launch<true> : rcell_launch<false>, rs, 8);
  }
  const bool chem = pc->chem == PGB_CHEM_COUPLED;
  if (chem) for_blocks(pc, R_INNER, rsource_launch, rs, 2);
  if (pc->visc) {
    for_blocks(pc, R_INNER, rgrads_launch, rs, 2);
    grads_fill(pc);
    mark(pc, 0);
  }
  for_blocks(pc, R_FX, rface_launch<0>, rs, 2);
  for_blocks(pc, R_FY, rface_launch<1>, rs, 2);
  for_blocks(pc, R_FZ, rface_launch<2>, rs, 2);
  RApplyCtx ra{};
  RApplyArgs &a = ra.a;
  a.dQ = rs->dQ;
  a.dt = pc->dt;
  a.chem = chem ? 1 : 0;
  a.write_dq = rs->write_dq;
  a.ncomb = rs->ncomb;
  a.comb[0] = rs->comb[0];
  a.comb[1] = rs->comb[1];
  for_blocks(pc, R_INNER, rapply_launch, &ra, 1);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "fused passes");
}

// the serving pool's reactors: one stage of every running reactor, and a
// reactor's state from its primitives
extern "C" int PGB_ENTRY(pgb_plain_reactors_)(const ReactorStage *rs, cudaStream_t s) {
  // a warp a reactor, eight a CTA
  if (rs->n > 0) k_reactors_warp<NS><<<(unsigned)((rs->n + 7) / 8), 256, 0, s>>>(*rs);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "reactors");
}

extern "C" int PGB_ENTRY(pgb_plain_reactor_prims_)(const double *prims, double *Q, double *T, int row,
                                                   long long cap, cudaStream_t s) {
  k_reactor_prims<NS><<<1, 1, 0, s>>>(prims, Q, T, row, cap);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "reactor primitives");
}
