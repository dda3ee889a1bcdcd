// pgb_rhs_block_noalloc: the right-hand side of one block with no device
// allocation at all.
//
// Who needs it: a caller that may not call cudaMalloc, or any routine that
// allocates device memory (torch's caching allocator included): code running
// inside another framework's memory pool or a fixed arena, or a solver
// embedded in a host application that owns all device memory.  The case API
// (pgb_case_finalize) allocates its registers, metrics and scratch; this call
// takes the caller's input and output arrays and keeps its scratch in a
// static device array instead.
//
// What it computes: the per-block path of pgb_rhs for one block whose halo
// the caller has filled (two layers on every face, the first layer of every
// edge): fromQ, transport, the cell gradients on the interior and the first
// halo layer (so no gradient exchange is needed), the advective and diffusive
// face fluxes of the three axes, and dQ.  The scratch it works in (the state,
// transport properties, species enthalpies, gradients and face fluxes) is the
// file-scope array below, of fixed size; every GPU that loads the library
// holds it until the process exits.  Every scratch value is written before
// it is read within one call, so nothing needs clearing; the array keeps the
// last call's contents.  All calls share the one array, and the species
// constants each call copies into this file's constant memory, so calls whose
// work overlaps on the GPU (two streams, two host threads) race on both and
// give wrong results: keep them ordered on one stream.
#include <mutex>
#include <string>

#include "pgb200.h"

// This unit's kernels under a name of their own.  The per-species units
// instantiate the same templates (k_fromQ<1>, k_advflux<2, 0>, ...), each
// against its own unit's constant memory; under one name the linker keeps
// one host launch stub for both, and a launch from either unit may run the
// other's copy, which reads the other unit's species constants.
#define pgb pgb_noalloc_unit
#include "plain.cuh"

using namespace pgb;

namespace {

// 2^21 doubles, 16 MiB: a block of up to (2^21 - 32) / (32 + 8 ns) cells
// halo included, 52,428 for one species (32^3 cells with their halo of two).
// Per cell: the state's 8 fields and the real gas's Z plane the transport
// kernel reads beside them (kept so no two of its arrays overlap), the
// transport properties (2 + ns), the species enthalpies (ns), the gradients
// (3 (ne - 1)) and the three axes' face fluxes (3 ne).
constexpr long long kScratchDoubles = 1ll << 21;
constexpr long long kHeadDoubles = 32;  // the block descriptor, 256 bytes
constexpr long long kStatePlanes = ST_Z + 1;
constexpr long long per_cell(int ns) { return kStatePlanes + (2 + ns) + ns + 3 * (3 + ns) + 3 * (4 + ns); }

static __device__ __align__(256) double g_scratch[kScratchDoubles];

// the array's device address, per device: looked up once, with that device
// current, on the first call there
std::mutex g_mutex;
double *g_addr[64] = {};

}  // namespace

// the library's error text (pgb_last_error), set from this file too
extern "C" int pgb_internal_fail(int code, const char *msg);

namespace {
int fail(int code, const std::string &msg) { return pgb_internal_fail(code, msg.c_str()); }
}  // namespace

extern "C" long long pgb_rhs_block_noalloc_max_cells(int ns) {
  if (ns < 1 || ns > MAXNS) return 0;
  return (kScratchDoubles - kHeadDoubles) / per_cell(ns);
}

extern "C" int pgb_rhs_block_noalloc(const pgb_physics *phys, const double *tables, int nx, int ny, int nz,
                                     const double *Q, const double *met, double *dQ, void *stream) {
  if (!phys || !tables || !Q || !met || !dQ) return fail(PGB_ERR_ARG, "null argument");
  const int ns = phys->ns;
  if (ns < 1 || ns > 3) return fail(PGB_ERR_UNSUPPORTED, "one to three species");
  if (phys->simulator != PGB_EULER && phys->simulator != PGB_NAVIER_STOKES)
    return fail(PGB_ERR_UNSUPPORTED, "the euler or navier-stokes simulator");
  if (phys->eos != PGB_EOS_CPG || phys->primary != PGB_FLUX_KEPAEC || phys->recon != PGB_RECON_CONSTANT)
    return fail(PGB_ERR_UNSUPPORTED, "the calorically perfect gas with kepaec on the cells as they are");
  const bool visc = phys->simulator == PGB_NAVIER_STOKES;
  if (visc && phys->trans != PGB_TRANS_CONSTANT) return fail(PGB_ERR_UNSUPPORTED, "constant transport only");
  if (phys->chemistry != PGB_CHEM_NONE) return fail(PGB_ERR_UNSUPPORTED, "no chemistry");
  if (nx < 2 || ny < 2 || nz < 2) return fail(PGB_ERR_ARG, "a block has at least two cells per axis");
  const long long X = nx + 2 * NG, Y = ny + 2 * NG, Z = nz + 2 * NG, V = X * Y * Z;
  const int ne = 4 + ns;
  const long long need = kHeadDoubles + V * per_cell(ns);
  if (need > kScratchDoubles)
    return fail(PGB_ERR_ARG, "block too large for the no-allocation scratch: at most " +
                                 std::to_string(pgb_rhs_block_noalloc_max_cells(ns)) +
                                 " cells halo included, this block has " + std::to_string(V));
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return fail(PGB_ERR_ARG, "device ordinal past 63");
  double *base;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_addr[dev]) {
      // the host's name for the array is not a device address: ask for it
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addr[dev] = (double *)p;
    }
    base = g_addr[dev];
  }
  // the species constants, packed: Rsp, cp0, h298R, MWinv, hpoly0, h298, mu0,
  // kappa0, MWqinv, lewis (ns each), then wilkepair (ns x ns)
  Species sp{};
  const double *tab[T_NTAB];
  for (int q = 0; q < T_NTAB; q++) tab[q] = tables + (long)q * ns;
  species_fill(sp, ns, phys->alpha, phys->trans == PGB_TRANS_CONSTANT, tab, tables + (long)T_NTAB * ns);
  e = cudaMemcpyToSymbolAsync(kSp, &sp, sizeof(Species), 0, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("species constants: ") + cudaGetErrorString(e));
  // the block's descriptor at the array's head (one block, starting at cell 0)
  BlockDev bd{};
  bd.nx = nx, bd.ny = ny, bd.nz = nz;
  bd.X = (int)X, bd.Y = (int)Y, bd.Z = (int)Z;
  bd.vol = V;
  bd.cv = 0;
  static_assert(sizeof(BlockDev) <= kHeadDoubles * sizeof(double), "descriptor fits the head");
  e = cudaMemcpyAsync(base, &bd, sizeof(BlockDev), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("block descriptor: ") + cudaGetErrorString(e));
  const BlockDev *blks = (const BlockDev *)base;
  double *state = base + kHeadDoubles;
  double *tr = state + kStatePlanes * V;
  double *hsp = tr + (2 + ns) * V;
  double *grads = hsp + ns * V;
  double *F[3];
  F[0] = grads + 3 * (ne - 1) * V;
  F[1] = F[0] + ne * V;
  F[2] = F[1] + ne * V;
  const int TH = 256;
  auto grid = [&](long long n) { return (unsigned)((n + TH - 1) / TH); };
  const long long inner = (long long)nx * ny * nz, shallow = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  const long long fx = (long long)(nx + 1) * ny * nz, fy = (long long)nx * (ny + 1) * nz, fz = (long long)nx * ny * (nz + 1);
#define PGB_NOALLOC_RHS(NS)                                                                               \
  k_fromQ<NS><<<grid(V), TH, 0, s>>>(blks, 0, Q, state);                                                  \
  if (visc) {                                                                                             \
    k_transport<NS><<<grid(V), TH, 0, s>>>(blks, 0, Q, state, tr, hsp);                                   \
    k_grads<NS><<<grid(shallow), TH, 0, s>>>(blks, 0, Q, state, met, grads, 1);                           \
  }                                                                                                       \
  k_advflux<NS, 0><<<grid(fx), TH, 0, s>>>(blks, 0, Q, state, met, F[0]);                                 \
  k_advflux<NS, 1><<<grid(fy), TH, 0, s>>>(blks, 0, Q, state, met, F[1]);                                 \
  k_advflux<NS, 2><<<grid(fz), TH, 0, s>>>(blks, 0, Q, state, met, F[2]);                                 \
  if (visc) {                                                                                             \
    k_diffflux<NS, 0><<<grid(fx), TH, 0, s>>>(blks, 0, Q, state, tr, hsp, grads, met, F[0]);              \
    k_diffflux<NS, 1><<<grid(fy), TH, 0, s>>>(blks, 0, Q, state, tr, hsp, grads, met, F[1]);              \
    k_diffflux<NS, 2><<<grid(fz), TH, 0, s>>>(blks, 0, Q, state, tr, hsp, grads, met, F[2]);              \
  }                                                                                                       \
  k_applyflux<NS><<<grid(inner), TH, 0, s>>>(blks, 0, F[0], F[1], F[2], met, dQ);
  switch (ns) {
    case 1: PGB_NOALLOC_RHS(1) break;
    case 2: PGB_NOALLOC_RHS(2) break;
    default: PGB_NOALLOC_RHS(3) break;
  }
#undef PGB_NOALLOC_RHS
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return PGB_OK;
}
