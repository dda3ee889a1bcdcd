// The per-block path for one species count, PGB_NS (1 when unset): the
// reference's passes one by one, one launch per block and kernel, each pass a
// round trip through HBM as in the reference's rhs graph
// (peregrine/simulator/advec/simulator.py:57-87,
// peregrine/simulator/advecdiff/simulator.py:110-124), with the coupled
// chemistry source beginning dQ (peregrine/simulator/chemint/coupled.py).
// The build compiles this file once per species count.
#include <algorithm>
#include <string>

#include "chem.cuh"
#include "pgb200.h"
#include "plain.cuh"
#include "plain_api.h"

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

int cuda_fail(cudaError_t e, const char *what) {
  return pgb_internal_fail(e == cudaErrorMemoryAllocation ? PGB_ERR_NOMEM : PGB_ERR_CUDA,
                           (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

void mark(const PlainCase *pc, int kind) {
  if (pc->mark) pc->mark(pc->ctx, kind);
}

template <int A, int FN>
void launch_riemann(const PlainCase *pc, int b, const double *Q, long long nf) {
  const int lim = pc->recon == PGB_RECON_MUSCL ? pc->limiter : 0;
  k_riemann<NS, A, FN><<<grid_of(nf), TH, 0, pc->stream>>>(pc->d_blks, b, Q, pc->state, pc->met, pc->F[A], lim);
}

template <int A>
void launch_advflux(const PlainCase *pc, int b, const double *Q, long long nf) {
  switch (pc->primary) {
    case PGB_FLUX_HLLC: launch_riemann<A, FN_HLLC>(pc, b, Q, nf); break;
    case PGB_FLUX_RUSANOV: launch_riemann<A, FN_RUSANOV>(pc, b, Q, nf); break;
    case PGB_FLUX_AUSMUP: launch_riemann<A, FN_AUSMUP>(pc, b, Q, nf); break;
    default: k_advflux<NS, A><<<grid_of(nf), TH, 0, pc->stream>>>(pc->d_blks, b, Q, pc->state, pc->met, pc->F[A]);
  }
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
  }
  if (mt) {
    e = cudaMemcpyToSymbolAsync(gMath, mt, sizeof(MathTables), 0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "math tables");
  }
  return PGB_OK;
}

// one right-hand side of every block: Q's halo, the state everywhere (the
// transport and gradients on the viscous path, the gradients' first halo
// layer), the chemistry source, the face fluxes per axis and the divergence
extern "C" int PGB_ENTRY(pgb_plain_rhs_)(const PlainCase *pc, const double *Q, double *dQ) {
  cudaStream_t s = pc->stream;
  double *Qm = const_cast<double *>(Q);
  k_halo<<<grid_of(pc->nhalo), TH, 0, s>>>(Qm, pc->halo, pc->nhalo, NE);
  mark(pc, 0);
  for (int b = 0; b < pc->nblocks; b++) {
    const BlockDev &D = pc->h_blks[b];
    const long long inner = (long long)D.nx * D.ny * D.nz;
    k_fromQ<NS><<<grid_of(D.vol), TH, 0, s>>>(pc->d_blks, b, Q, pc->state);
    mark(pc, 2);
    if (pc->visc) {
      k_transport<NS><<<grid_of(D.vol), TH, 0, s>>>(pc->d_blks, b, Q, pc->state, pc->tr, pc->hsp);
      mark(pc, 2);
      k_grads<NS><<<grid_of(inner), TH, 0, s>>>(pc->d_blks, b, Q, pc->state, pc->met, pc->grads);
      mark(pc, 2);
    }
  }
  if (pc->visc) {
    k_halo<<<grid_of(pc->nhalo_l0), TH, 0, s>>>(pc->grads, pc->halo, pc->nhalo_l0, 3 * (NE - 1));
    mark(pc, 0);
  }
  for (int b = 0; b < pc->nblocks; b++) {
    const BlockDev &D = pc->h_blks[b];
    const long long inner = (long long)D.nx * D.ny * D.nz;
    const long long fx = (long long)(D.nx + 1) * D.ny * D.nz, fy = (long long)D.nx * (D.ny + 1) * D.nz,
                    fz = (long long)D.nx * D.ny * (D.nz + 1);
    if (pc->chem) {
      k_source<NS><<<grid_of(inner), TH, 0, s>>>(pc->d_blks, b, Q, pc->state, dQ);
      mark(pc, 2);
    }
    launch_advflux<0>(pc, b, Q, fx);
    mark(pc, 2);
    launch_advflux<1>(pc, b, Q, fy);
    mark(pc, 2);
    launch_advflux<2>(pc, b, Q, fz);
    mark(pc, 2);
    if (pc->visc) {
      k_diffflux<NS, 0><<<grid_of(fx), TH, 0, s>>>(pc->d_blks, b, Q, pc->state, pc->tr, pc->hsp, pc->grads, pc->met, pc->F[0]);
      mark(pc, 2);
      k_diffflux<NS, 1><<<grid_of(fy), TH, 0, s>>>(pc->d_blks, b, Q, pc->state, pc->tr, pc->hsp, pc->grads, pc->met, pc->F[1]);
      mark(pc, 2);
      k_diffflux<NS, 2><<<grid_of(fz), TH, 0, s>>>(pc->d_blks, b, Q, pc->state, pc->tr, pc->hsp, pc->grads, pc->met, pc->F[2]);
      mark(pc, 2);
    }
    k_applyflux<NS><<<grid_of(inner), TH, 0, s>>>(pc->d_blks, b, pc->F[0], pc->F[1], pc->F[2], pc->met, dQ, pc->chem);
    mark(pc, 2);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PGB_OK : cuda_fail(e, "per-block launch");
}

// Q and the state of one block's interior from its primitives
extern "C" int PGB_ENTRY(pgb_plain_fromprims_)(const PlainCase *pc, int blk, const double *prims, double *Q) {
  const BlockDev &D = pc->h_blks[blk];
  k_fromprims<NS><<<grid_of((long long)D.nx * D.ny * D.nz), TH, 0, pc->stream>>>(pc->d_blks, blk, prims, Q, pc->state);
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
