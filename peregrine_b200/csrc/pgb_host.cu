// The host side of pgb200: cases, device arrays, halo tables, the stage plans
// and the launches, behind the C ABI of include/pgb200.h.
#include "pgb200.h"
#include "rategen.h"

#include <algorithm>
#include <cstddef>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "fused.cuh"
#include "fused2.cuh"
#include "fused3.cuh"
#include "layout.cuh"
#include "physics.cuh"
#include "plain.cuh"
#include "plain_api.h"

using namespace pgb;

PGB_PLAIN_DECL(1)
PGB_PLAIN_DECL(2)
PGB_PLAIN_DECL(3)
PGB_PLAIN_DECL(4)
PGB_PLAIN_DECL(5)
PGB_PLAIN_DECL(6)
PGB_PLAIN_DECL(7)
PGB_PLAIN_DECL(8)
PGB_PLAIN_DECL(9)
PGB_PLAIN_DECL(10)
PGB_PLAIN_DECL(11)
PGB_PLAIN_DECL(12)

namespace {
#define PGB_OPS(N)                                                                                          \
  {pgb_plain_upload_##N, pgb_plain_rhs_##N, pgb_plain_fromprims_##N, pgb_plain_production_##N, pgb_plain_prestep_##N, \
   pgb_plain_cflmax_##N, pgb_plain_fused_##N, pgb_plain_reactors_##N, pgb_plain_reactor_prims_##N}
// the per-block path of each species count, 1 to MAXNS
const PlainOps kPlain[MAXNS] = {PGB_OPS(1), PGB_OPS(2), PGB_OPS(3), PGB_OPS(4),  PGB_OPS(5),  PGB_OPS(6),
                                PGB_OPS(7), PGB_OPS(8), PGB_OPS(9), PGB_OPS(10), PGB_OPS(11), PGB_OPS(12)};
#undef PGB_OPS
}  // namespace

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? PGB_ERR_NOMEM : PGB_ERR_CUDA,            \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

#define RET(call)             \
  do {                        \
    int r_ = (call);          \
    if (r_ != PGB_OK) return r_; \
  } while (0)

static __global__ void k_setscalar(double *p, double v) { *p = v; }
// a shard's halo cells to and from a buffer [component][cell]: cell e's
// component c at R[at[e] + c vol[e]]
static __global__ void k_xpack(const double *__restrict__ R, const long long *__restrict__ at,
                               const int *__restrict__ vol, long long n, int ne, double *__restrict__ buf) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < ne; c++) buf[c * n + e] = R[at[e] + (long long)c * vol[e]];
}
static __global__ void k_xunpack(double *__restrict__ R, const long long *__restrict__ at,
                                 const int *__restrict__ vol, long long n, int ne, const double *__restrict__ buf) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < ne; c++) R[at[e] + (long long)c * vol[e]] = buf[c * n + e];
}
// the clock at a step's end: start + dt (peregrine/multiblock/solver.py:355-364)
static __global__ void k_clock(double *clock, const double *dt) { *clock = *clock + *dt; }
// the cfl controller's step: min(cfl / the combined CFL number per unit step,
// dt-max), ctrl = {cfl, dt-max} (peregrine/integrators/controllers.py:21-30)
static __global__ void k_cfldt(double *dt, const double *cfl, const double *ctrl) {
  *dt = fmin(ctrl[0] / cfl[2], ctrl[1]);
}

struct HostBlock {
  int nx, ny, nz;
  int nbr[6] = {-1, -1, -1, -1, -1, -1};
  int nbrface[6] = {0, 0, 0, 0, 0, 0};
  // per face, the reference's orientation digits: for each of this block's
  // axes the neighbour's axis it runs along, 1-3 forward, 4-6 backward
  int orient[6][3] = {{1, 2, 3}, {1, 2, 3}, {1, 2, 3}, {1, 2, 3}, {1, 2, 3}, {1, 2, 3}};
  int rot[6] = {0, 0, 0, 0, 0, 0};  // a rotationally periodic face's rotation, 1 + its index
  int bc[6] = {-1, -1, -1, -1, -1, -1};  // a boundary face's entry, -1 for none
  int tw = 0, th = 0, kchunk = 0;
  bool metrics_set[PGB_NMETRICS] = {};
  BlockDev dev{};
};

// a stage's launch plan on the fused path, physical registers resolved: the
// register the stage reads, the buffer dQ's logical register names at the
// stage's start (the fused passes' source lands there), the combines
struct FusedStagePlan {
  int qin;
  int dqbuf;
  int ncomb;
  FusedCombine comb[2];
};

}  // namespace

struct pgb_case {
  pgb_physics phys{};
  Species sp{};
  std::map<std::string, std::vector<double>> tables;
  std::vector<HostBlock> blocks;
  std::vector<pgb_stage> stages;
  bool finalized = false;
  int ne = 5;
  long long cells = 0;  // total cells, halo included
  // device
  cudaStream_t stream = nullptr;
  BlockDev *d_blks = nullptr;
  double *d_reg[MAXREGS] = {};
  double *d_met = nullptr;
  double *d_dt = nullptr;
  double *d_one = nullptr;  // 1.0: the step size of a right-hand side on the fused path
  HaloEntry *d_halo = nullptr;
  long long nhalo = 0, nhalo_l0 = 0;  // all entries; face layer 0 only (first)
  // the same halo as boxes (k_halo_boxes): the boxes, the CTA table and the
  // cells no box holds, listed one by one
  HaloPatch *d_boxes = nullptr;
  int2 *d_boxcta = nullptr;
  HaloEntry *d_boxrest = nullptr;
  long long nboxcta = 0, nboxrest = 0;
  // the rotationally periodic faces' rotations, then the products a halo
  // cell reached across two of them needs, 3 x 3 each
  std::vector<double> rots;
  double *d_rots = nullptr;
  // per-block path scratch
  double *d_state = nullptr, *d_tr = nullptr, *d_hsp = nullptr, *d_grads = nullptr, *d_F[3] = {};
  double *d_prims = nullptr;
  long long prims_cap = 0;
  // fused path
  TileDev *d_tiles = nullptr;
  int ntiles = 0;
  unsigned int *d_counter = nullptr;
  size_t fused_smem = 0;
  bool tiles_dirty = true;
  bool uniform_done = false;
  bool use_v2 = false;  // every block uniform: the uniform-metric fused kernel
  int form = 0;         // the batched path's form: 1 the fused stage kernel, 2 the fused passes
  // a shard's exchange with the other ranks' blocks: the cells it packs and
  // unpacks, each its component 0's offset in a register and its component stride
  long long *d_xsend = nullptr, *d_xrecv = nullptr;
  int *d_xsvol = nullptr, *d_xrvol = nullptr;
  long long nxsend = 0, nxrecv = 0;
  int stage_next = 0;  // the next stage pgb_step_stage runs

  int v2_ctas = 1;      // its resident CTAs per SM
  int v2 = 0;           // its instance: threads per CTA, launch bound, tile layout
  // the uniform stage reads across faces from the neighbours' cells in place
  // of a halo fill: wanted (the default), and whether every face allows it
  bool pull_want = true, pull_faces = false;
  int *d_nbr27 = nullptr;  // per block, the block one step away along each axis
  // register mapping: logical -> physical
  std::vector<int> phys_of, canonical;
  int period = 1, phase = 0;
  std::vector<std::vector<FusedStagePlan>> plans;  // [phase][stage]
  std::vector<std::vector<int>> maps;              // mapping at the start of each phase
  // graphs
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  std::vector<int> graph_map[3];  // the mapping a graph was captured under
  bool packed = false;            // the per-block kernels, each pass one launch over every block
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.0f;
  int launches[3] = {0, 0, 0};
  // per-launch timing (pgb_step_timed): an event after every launch
  bool timing = false;
  std::vector<cudaEvent_t> tev;
  std::vector<int> tkind;
  size_t tnext = 0;
  double *d_stage = nullptr;  // whole-state staging
  long long stage_cap = 0;
  // finite-rate chemistry: the mechanism's device tables
  std::unique_ptr<Mech> mech;
  // the finite-rate source generated for the mechanism (rategen.cu): wanted
  // (the default), its loaded library and kernel, the table log's and exp's
  // tables it reads, and why it is not in use when it is not
  bool gen_want = true;
  cudaLibrary_t gen_lib = nullptr;
  const void *gen_src = nullptr;
  MathTables *d_math = nullptr;
  std::string gen_why;
  unsigned long long uid = 0;  // unique over the process, never reused
  unsigned version = 0;        // bumped when the species or mechanism tables change
  bool df_fresh = true;        // the double flux has no frozen planes for the state yet
  bool state_stale = false;    // a batched step since the state array was last written
  // boundaries: the entries and their programs as given, then on the device
  // the entries, programs and the three passes' face tables (each with its
  // sentinel), and the clock the boundary values read
  std::vector<BcEntry> bc_entries;
  std::vector<BcOp> bc_ops;
  BcEntry *d_bcent = nullptr;
  BcOp *d_bcops = nullptr;
  BcFace *d_bcface[3] = {};  // halo, gradient and wall passes
  int nbcface[3] = {0, 0, 0};
  long long bcthreads[3] = {0, 0, 0};
  double *d_clock = nullptr;
  // the cfl controller: its reduction's three maxima, its {cfl, dt-max}, whether
  // the steps run under it, and the mode each path's graph was captured in
  double *d_cfl = nullptr, *d_ctrl = nullptr;
  bool ctrl_cfl = false;
  bool graph_cfl[3] = {false, false, false};
  // the sub-stepped chemistry: its options, each cell's last count, the stiff list
  SubstepOpts subopt{200, 1, 8, 1e-7, 1e-12, 1.0, 0.0};
  int *d_subs = nullptr;
  unsigned int *d_stiffhead = nullptr;
  int2 *d_stiffcells = nullptr;
  long long interior_cells = 0;
};

namespace {

// the simulators' two traits: viscous (navier-stokes, navier-stokes-df) and
// the double flux (euler-df, navier-stokes-df)
inline bool sim_visc(int s) { return s == PGB_NAVIER_STOKES || s == PGB_NAVIER_STOKES_DF; }
inline bool sim_df(int s) { return s == PGB_EULER_DF || s == PGB_NAVIER_STOKES_DF; }

// The batched path's form for a case: 1, the fused stage kernel (the
// calorically perfect single-species gas, kepaec on the cells as they are,
// inviscid or with constant transport); 2, the fused passes (any other ideal
// gas, flux function and reconstruction, inviscid or viscous, with or without
// the coupled chemistry source); 0, neither (boundaries, the real gas, the
// double flux, the sub-stepped chemistry: the per-block kernels, packed).
int batched_form(const pgb_case *c) {
  const pgb_physics &p = c->phys;
  // the batched kernels' halo is the periodic or block-to-block fill alone,
  // and their tiles and stencil take blocks of two cells or more per axis
  for (const HostBlock &B : c->blocks) {
    if (B.nx < 2 || B.ny < 2 || B.nz < 2) return 0;
    for (int f = 0; f < 6; f++)
      if (B.bc[f] >= 0) return 0;
  }
  // the double flux's inviscid kepaec case: the fused passes' cell-centric stage
  if (p.simulator == PGB_EULER_DF)
    return p.eos == PGB_EOS_REALGAS_DF && p.primary == PGB_FLUX_KEPAEC && p.recon == PGB_RECON_CONSTANT ? 2 : 0;
  if (p.simulator != PGB_EULER && p.simulator != PGB_NAVIER_STOKES) return 0;
  if (p.eos != PGB_EOS_CPG && p.eos != PGB_EOS_TPG) return 0;
  if (p.chemistry == PGB_CHEM_SUBSTEPPED) return 0;
  if (p.eos == PGB_EOS_CPG && p.primary == PGB_FLUX_KEPAEC && p.recon == PGB_RECON_CONSTANT && p.ns == 1 &&
      (p.simulator == PGB_EULER || p.trans == PGB_TRANS_CONSTANT))
    return 1;
  return 2;
}
bool fused_capable(const pgb_case *c) { return batched_form(c) > 0; }

const double *table(const pgb_case *c, const char *name) {
  auto it = c->tables.find(name);
  return it == c->tables.end() ? nullptr : it->second.data();
}

// the case's named species tables into the constant struct
int build_species(pgb_case *c) {
  const int ns = c->phys.ns;
  static const char *names[T_NTAB] = {"Rsp", "cp0", "h298R", "MWinv", "hpoly0", "h298", "mu0", "kappa0", "MWqinv", "lewis"};
  // cp0 is the calorically perfect gas's; the thermally perfect one reads its fits
  const bool cpg = c->phys.eos == PGB_EOS_CPG;
  const bool need[T_NTAB] = {true, cpg, true, true, false, false, false, false, false, false};
  const double *tab[T_NTAB];
  for (int q = 0; q < T_NTAB; q++) {
    tab[q] = table(c, names[q]);
    if (!tab[q] && need[q]) return fail(PGB_ERR_ARG, std::string("species table ") + names[q] + " not set");
    if (tab[q] && (long)c->tables[names[q]].size() < ns)
      return fail(PGB_ERR_ARG, std::string("species table ") + names[q] + " short");
  }
  if (c->phys.trans == PGB_TRANS_CONSTANT && (!tab[T_MU0] || !tab[T_KAPPA0]))
    return fail(PGB_ERR_ARG, "constant transport needs mu0 and kappa0");
  species_fill(c->sp, ns, c->phys.alpha, c->phys.trans == PGB_TRANS_CONSTANT, tab, table(c, "wilkepair"));
  // the thermally perfect fits and the kinetic-theory fits, [ns][terms]
  auto fit = [&](const char *name, double *dst, int &terms) -> int {
    auto it = c->tables.find(name);
    if (it == c->tables.end()) return fail(PGB_ERR_ARG, std::string("table ") + name + " not set");
    const long n = (long)it->second.size();
    if (n % ns || n / ns < 1 || n / ns > MAXT)
      return fail(PGB_ERR_ARG, std::string("table ") + name + ": species times 1 to 8 terms");
    fit_fill(dst, terms, it->second.data(), ns, (int)(n / ns));
    return PGB_OK;
  };
  if (c->phys.eos != PGB_EOS_CPG) {
    c->sp.tpg = 1;
    RET(fit("cppolyR", c->sp.cppolyR, c->sp.ncp));
    RET(fit("hpoly", c->sp.hpoly, c->sp.nh));
  }
  if (c->phys.eos == PGB_EOS_REALGAS || c->phys.eos == PGB_EOS_REALGAS_DF) {
    c->sp.realgas = 1;
    c->sp.df = c->phys.eos == PGB_EOS_REALGAS_DF;
    struct {
      const char *name;
      double *dst;
    } one[] = {{"cubicu", &c->sp.cu}, {"cubicw", &c->sp.cw}, {"cubicsigma", &c->sp.csigma}, {"cubiceps", &c->sp.ceps}};
    for (auto &t : one) {
      const double *v = table(c, t.name);
      if (!v) return fail(PGB_ERR_ARG, std::string("real-gas table ") + t.name + " not set");
      *t.dst = v[0];
    }
    struct {
      const char *name;
      double *dst;
    } per[] = {{"cubicsqrtac", c->sp.csqrtac}, {"cubicb", c->sp.cb}, {"cubicda", c->sp.cda},
               {"cubicmTc", c->sp.cmTc}, {"cubiconepm", c->sp.conepm}, {"vshift", c->sp.vshift},
               {"cubicsqrtacMW", c->sp.csqrtacMW}, {"cubicbMW", c->sp.cbMW}, {"cubicdaMW", c->sp.cdaMW},
               {"vshiftMW", c->sp.vshiftMW}};
    for (auto &t : per) {
      auto it = c->tables.find(t.name);
      if (it == c->tables.end() || (long)it->second.size() < ns)
        return fail(PGB_ERR_ARG, std::string("real-gas table ") + t.name + " not set or short");
      for (int n = 0; n < ns; n++) t.dst[n] = it->second[n];
    }
  }
  if (c->phys.trans == PGB_TRANS_KINETIC) {
    c->sp.kinetic = 1;
    RET(fit("mupoly", c->sp.mupoly, c->sp.nmu));
    RET(fit("kappapoly", c->sp.kappapoly, c->sp.nkappa));
  }
  // Herning's mixing rule, when its sqrt(MW) are given
  c->sp.herning = 0;
  if (const double *sq = table(c, "sqrtMW")) {
    if ((long)c->tables["sqrtMW"].size() < ns) return fail(PGB_ERR_ARG, "sqrtMW short");
    for (int n = 0; n < ns; n++) c->sp.sqrtMW[n] = sq[n];
    c->sp.herning = 1;
  }
  // binary diffusion, when its pair fits are given: "selffit" [ns][terms],
  // "pairfit" [ns][width][terms], "bath" the species a partial bath sums over
  // (peregrine/simulator/mixture/diffusion/binary.py:18-37)
  c->sp.binary = 0;
  if (table(c, "pairfit") || table(c, "selffit")) {
    if (!table(c, "pairfit") || !table(c, "selffit")) return fail(PGB_ERR_ARG, "binary diffusion takes pairfit and selffit");
    const std::vector<double> &self = c->tables["selffit"], &pair = c->tables["pairfit"];
    if (self.size() % ns || self.size() / ns < 1 || self.size() / ns > MAXT)
      return fail(PGB_ERR_ARG, "selffit: species times 1 to 8 terms");
    const int terms = (int)(self.size() / ns);
    int width = ns - 1;
    c->sp.bpartial = 0;
    if (table(c, "bath")) {
      const std::vector<double> &bath = c->tables["bath"];
      if (bath.empty() || (int)bath.size() > ns) return fail(PGB_ERR_ARG, "bath: 1 to ns species");
      for (size_t k = 0; k < bath.size(); k++) {
        const int m = (int)bath[k];
        if (m < 0 || m >= ns || (double)m != bath[k]) return fail(PGB_ERR_ARG, "bath: species indices");
        c->sp.bath[k] = m;
      }
      if ((int)bath.size() < ns) c->sp.bpartial = 1, width = (int)bath.size();
    }
    if ((long)pair.size() != (long)ns * width * terms)
      return fail(PGB_ERR_ARG, "pairfit: species times partners times the selffit's terms");
    c->sp.bwidth = width, c->sp.npair = terms, c->sp.nself = terms;
    for (int n = 0; n < ns; n++)
      for (int t = 0; t < MAXT; t++) {
        c->sp.selffit[n * MAXT + t] = t < terms ? self[n * terms + t] : 0.0;
        for (int k = 0; k < MAXNS; k++)
          c->sp.pairfit[(n * MAXNS + k) * MAXT + t] = (k < width && t < terms) ? pair[(n * width + k) * terms + t] : 0.0;
      }
    const double *mw = table(c, "MW");
    if (!mw || (long)c->tables["MW"].size() < ns) return fail(PGB_ERR_ARG, "binary diffusion reads MW");
    for (int n = 0; n < ns; n++) c->sp.MW[n] = mw[n];
    c->sp.binary = 1;
  }
  if (c->phys.chemistry != PGB_CHEM_NONE && !c->mech)
    return fail(PGB_ERR_STATE, "finite-rate chemistry needs pgb_case_set_mechanism before finalize");
  if (c->phys.chemistry == PGB_CHEM_SUBSTEPPED) {
    // the integrator's cv and the exit's concentration floor read cp / R and the molar masses
    RET(fit("cppoly", c->sp.cppoly, c->sp.ncppoly));
    const double *mw = table(c, "MW");
    if (!mw || (long)c->tables["MW"].size() < ns) return fail(PGB_ERR_ARG, "the sub-stepped chemistry reads MW");
    for (int n = 0; n < ns; n++) c->sp.MW[n] = mw[n];
  }
  c->version++;
  return PGB_OK;
}

// which case's tables each species count's unit holds, so a case's repeated
// launches upload nothing
// The owner is the case (or pool) whose launches were queued last against
// the tables: its stream is where launches that read them may still be
// waiting.
struct Uploaded {
  unsigned long long uid = 0;
  unsigned version = 0;
  int device = -1;
  cudaStream_t stream = nullptr;
  bool same(unsigned long long id, unsigned ver, int dev) const { return uid == id && version == ver && device == dev; }
};
Uploaded g_host_up, g_plain_up[MAXNS];
unsigned long long g_next_uid = 0;

// A new owner's upload must not land while the previous owner's queued
// launches can still read the tables: the new owner's stream waits for an
// event marking everything the previous owner's stream holds now.  The
// previous owner, taking the tables back later, waits the same way.
int take_tables(Uploaded &u, unsigned long long id, unsigned ver, int dev, cudaStream_t to) {
  if (u.stream && u.device == dev && u.stream != to) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaError_t r = cudaEventRecord(e, u.stream);
    if (r == cudaSuccess) r = cudaStreamWaitEvent(to, e, 0);
    cudaEventDestroy(e);  // released once it completes
    if (r != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("table handover: ") + cudaGetErrorString(r));
  }
  u.uid = id, u.version = ver, u.device = dev, u.stream = to;
  return PGB_OK;
}

// a stream about to be destroyed (its work done) owns nothing any more
void forget_stream(cudaStream_t s) {
  if (g_host_up.stream == s) g_host_up.stream = nullptr;
  for (Uploaded &u : g_plain_up)
    if (u.stream == s) u.stream = nullptr;
}

int set_current(pgb_case *c) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (!g_host_up.same(c->uid, c->version, dev)) {
    RET(take_tables(g_host_up, c->uid, c->version, dev, c->stream));
    CK(cudaMemcpyToSymbolAsync(kSp, &c->sp, sizeof(Species), 0, cudaMemcpyHostToDevice, c->stream));
  } else if (g_host_up.stream != c->stream) {
    g_host_up.stream = c->stream;
  }
  Uploaded &u = g_plain_up[c->phys.ns - 1];
  if (!u.same(c->uid, c->version, dev)) {
    static MathTables mt;
    static bool filled = false;
    if (!filled) math_tables_fill(mt), filled = true;
    RET(take_tables(u, c->uid, c->version, dev, c->stream));
    RET(kPlain[c->phys.ns - 1].upload(&c->sp, c->mech.get(), c->mech ? &mt : nullptr, c->stream));
  }
  return PGB_OK;
}

// each block's extents and its cells' offset in a register, blocks end to
// end; returns the cells of them all
long long layout_blocks(pgb_case *c) {
  long long cv = 0;
  for (auto &B : c->blocks) {
    BlockDev &D = B.dev;
    D = BlockDev{};
    D.nx = B.nx, D.ny = B.ny, D.nz = B.nz;
    D.X = B.nx + 2 * NG, D.Y = B.ny + 2 * NG, D.Z = B.nz + 2 * NG;
    D.vol = (long long)D.X * D.Y * D.Z;
    D.cv = cv;
    cv += D.vol;
  }
  return cv;
}

// where a cell outside a block lies: step across the face of the first axis
// it lies outside of, into the neighbour's own axes by the face's
// orientation (the reference's digits, peregrine/multiblock/interface/base.py:96-160),
// as many times as a block thinner than the halo or an edge cell needs;
// false at a boundary.  rot: the rotation the cell's vectors take on the way
// (1 + its index in the case's table, 0 for none), the faces' own composed.
bool locate(pgb_case *c, int b, int ijk[3], int &sb, int &rot) {
  sb = b;
  rot = 0;
  for (int hop = 0; hop < 4 * (NG + 1); hop++) {
    const HostBlock &B = c->blocks[sb];
    const int n[3] = {B.nx, B.ny, B.nz};
    int a = -1;
    for (int d = 0; d < 3 && a < 0; d++)
      if (ijk[d] < 0 || ijk[d] >= n[d]) a = d;
    if (a < 0) return true;
    const bool low = ijk[a] < 0;
    const int f = 2 * a + (low ? 0 : 1);
    const int nb = B.nbr[f];
    if (nb < 0) return false;
    const HostBlock &N = c->blocks[nb];
    const int m[3] = {N.nx, N.ny, N.nz};
    int out[3];
    for (int d = 0; d < 3; d++) {
      const int t = (B.orient[f][d] - 1) % 3;
      const bool flip = B.orient[f][d] > 3;
      if (d == a) {
        // the depth past the face; the neighbour meets a low face with its
        // high one unless the axis runs backward
        const int depth = low ? -1 - ijk[a] : ijk[a] - n[a];
        const bool theirlow = low == flip;
        out[t] = theirlow ? depth : m[t] - 1 - depth;
      } else {
        out[t] = flip ? m[t] - 1 - ijk[d] : ijk[d];
      }
    }
    if (B.rot[f]) {
      if (!rot) {
        rot = B.rot[f];
      } else {
        // a cell across two rotating faces: the product, the nearer face's on the left
        const double *R1 = &c->rots[9 * (rot - 1)], *R2 = &c->rots[9 * (B.rot[f] - 1)];
        double P[9];
        for (int r = 0; r < 3; r++)
          for (int q = 0; q < 3; q++) P[3 * r + q] = R1[3 * r] * R2[q] + R1[3 * r + 1] * R2[3 + q] + R1[3 * r + 2] * R2[6 + q];
        c->rots.insert(c->rots.end(), P, P + 9);
        rot = (int)(c->rots.size() / 9);
      }
    }
    ijk[0] = out[0], ijk[1] = out[1], ijk[2] = out[2];
    sb = nb;
  }
  return false;
}

// every halo cell a stage reads: the face halos two deep (layer 0 of every
// face first, as the gradients' one-plane exchange reads only those), then
// the edge cells one deep in both axes
void build_halo(pgb_case *c, std::vector<HaloEntry> &out, long long &n_l0, std::vector<int2> *blocks = nullptr) {
  out.clear();
  if (blocks) blocks->clear();
  auto add = [&](int b, int i, int j, int k) {
    int ijk[3] = {i, j, k};
    int sb, rot;
    if (!locate(c, b, ijk, sb, rot)) return;
    const BlockDev &D = c->blocks[b].dev, &S = c->blocks[sb].dev;
    HaloEntry h;
    h.dcv = D.cv, h.scv = S.cv;
    h.didx = (int)cell_index(D, i + NG, j + NG, k + NG);
    h.sidx = (int)cell_index(S, ijk[0] + NG, ijk[1] + NG, ijk[2] + NG);
    h.dvol = (int)D.vol, h.svol = (int)S.vol;
    h.rot = rot;
    out.push_back(h);
    if (blocks) blocks->push_back(make_int2(b, sb));
  };
  for (int layer = 0; layer < NG; layer++) {
    for (int b = 0; b < (int)c->blocks.size(); b++) {
      const HostBlock &B = c->blocks[b];
      const int n[3] = {B.nx, B.ny, B.nz};
      for (int f = 0; f < 6; f++) {
        const int a = f / 2;
        const bool low = f % 2 == 0;
        const int x = low ? -1 - layer : n[a] + layer;
        // the lower tangential axis fastest, so neighbouring entries (threads)
        // touch neighbouring cells: i on the j- and k-faces, j on the i-faces
        const int a1 = a == 0 ? 1 : 0, a2 = a == 2 ? 1 : 2;
        for (int q2 = 0; q2 < n[a2]; q2++)
          for (int q1 = 0; q1 < n[a1]; q1++) {
            int ijk[3];
            ijk[a] = x, ijk[a1] = q1, ijk[a2] = q2;
            add(b, ijk[0], ijk[1], ijk[2]);
          }
      }
    }
    if (layer == 0) n_l0 = (long long)out.size();
  }
  for (int b = 0; b < (int)c->blocks.size(); b++) {
    const HostBlock &B = c->blocks[b];
    const int n[3] = {B.nx, B.ny, B.nz};
    for (int a = 0; a < 3; a++) {
      const int a1 = (a + 1) % 3, a2 = (a + 2) % 3;
      for (int s1 = 0; s1 < 2; s1++)
        for (int s2 = 0; s2 < 2; s2++)
          for (int q = 0; q < n[a]; q++) {
            int ijk[3];
            ijk[a] = q;
            ijk[a1] = s1 ? n[a1] : -1;
            ijk[a2] = s2 ? n[a2] : -1;
            add(b, ijk[0], ijk[1], ijk[2]);
          }
    }
  }
}

// The halo as boxes: each face's halo NG deep and each edge line one deep,
// the cells build_halo lists, as a box wherever one block holds every cell's
// source and the source index is affine in the cell's (a face whose
// neighbour is at least NG cells thick, an edge line along a block); the
// cells of any other box are listed one by one in rest.
void build_boxes(pgb_case *c, std::vector<HaloPatch> &boxes, std::vector<HaloEntry> &rest) {
  boxes.clear();
  rest.clear();
  auto box = [&](int b, const int lo[3], const int hi[3]) {
    const BlockDev &D = c->blocks[b].dev;
    const int n[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
    std::vector<HaloEntry> es;
    bool all = true;
    for (int k = lo[2]; k < hi[2]; k++)
      for (int j = lo[1]; j < hi[1]; j++)
        for (int i = lo[0]; i < hi[0]; i++) {
          int ijk[3] = {i, j, k};
          int sb, rot;
          if (!locate(c, b, ijk, sb, rot)) {
            all = false;
            continue;
          }
          const BlockDev &S = c->blocks[sb].dev;
          HaloEntry h;
          h.dcv = D.cv, h.scv = S.cv;
          h.didx = (int)cell_index(D, i + NG, j + NG, k + NG);
          h.sidx = (int)cell_index(S, ijk[0] + NG, ijk[1] + NG, ijk[2] + NG);
          h.dvol = (int)D.vol, h.svol = (int)S.vol;
          h.rot = rot;
          es.push_back(h);
        }
    if (es.empty()) return;
    bool affine = all;
    HaloPatch P{};
    if (affine) {
      const HaloEntry &e0 = es[0];
      P.dcv = e0.dcv, P.scv = e0.scv, P.dvol = e0.dvol, P.svol = e0.svol, P.rot = e0.rot;
      P.d0 = e0.didx, P.s0 = e0.sidx;
      const int step[3] = {1, n[0], n[0] * n[1]};
      for (int d = 0; d < 3; d++) {
        P.dst[d] = n[d] > 1 ? es[step[d]].didx - e0.didx : 0;
        P.sst[d] = n[d] > 1 ? es[step[d]].sidx - e0.sidx : 0;
      }
      P.n0 = n[0], P.n1 = n[1], P.cells = n[0] * n[1] * n[2];
      size_t e = 0;
      for (int k = 0; k < n[2] && affine; k++)
        for (int j = 0; j < n[1] && affine; j++)
          for (int i = 0; i < n[0] && affine; i++, e++) {
            const HaloEntry &h = es[e];
            affine = h.scv == P.scv && h.svol == P.svol && h.rot == P.rot &&
                     h.didx == P.d0 + i * P.dst[0] + j * P.dst[1] + k * P.dst[2] &&
                     h.sidx == P.s0 + i * P.sst[0] + j * P.sst[1] + k * P.sst[2];
          }
    }
    if (affine)
      boxes.push_back(P);
    else
      rest.insert(rest.end(), es.begin(), es.end());
  };
  for (int b = 0; b < (int)c->blocks.size(); b++) {
    const HostBlock &B = c->blocks[b];
    const int n[3] = {B.nx, B.ny, B.nz};
    for (int f = 0; f < 6; f++) {
      const int a = f / 2;
      int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
      lo[a] = f % 2 == 0 ? -NG : n[a];
      hi[a] = lo[a] + NG;
      box(b, lo, hi);
    }
    for (int a = 0; a < 3; a++) {
      const int a1 = (a + 1) % 3, a2 = (a + 2) % 3;
      for (int s1 = 0; s1 < 2; s1++)
        for (int s2 = 0; s2 < 2; s2++) {
          int lo[3], hi[3];
          lo[a] = 0, hi[a] = n[a];
          lo[a1] = s1 ? n[a1] : -1, hi[a1] = lo[a1] + 1;
          lo[a2] = s2 ? n[a2] : -1, hi[a2] = lo[a2] + 1;
          box(b, lo, hi);
        }
    }
  }
}

int grid_for(long long n, int threads);

// the full halo of a register, comps components, vec the component its
// rotations turn: by the boxes when the case has them, else by entries
void halo_fill_case(pgb_case *c, double *base, int comps, int vec) {
  if (c->nboxcta > 0)
    halo_boxes_launch<5, SW>((unsigned)c->nboxcta, c->stream, base, c->d_boxes, c->d_boxcta, c->d_boxrest,
                               c->nboxrest, comps, vec, c->d_rots);
  else
    k_halo<<<grid_for(c->nhalo, 256), 256, 0, c->stream>>>(base, c->d_halo, c->nhalo, comps, vec, c->d_rots);
}

// the default tile of a block: a width that cuts i evenly in pieces of at
// most 32, as many rows as 128 threads allow, k cut in two runs
void default_tile(HostBlock &B) {
  const int pi = (B.nx + 31) / 32;
  int tw = (B.nx + pi - 1) / pi;
  int th = std::max(1, FUSED_THREADS / tw);
  th = std::min(th, B.ny);
  const int pj = (B.ny + th - 1) / th;
  th = (B.ny + pj - 1) / pj;
  B.tw = tw, B.th = th;
  B.kchunk = (B.nz + 1) / 2;
}

// The uniform kernel's instances: threads per CTA, the CTAs per SM its
// registers are bounded for, and the largest tile its shared layout holds.
struct V2Inst {
  int nt, minb, tw, th;
  const void *fvisc, *feuler;
  size_t smvisc, smeuler;
  bool pull;  // reads across faces from the neighbours' cells when the case allows
};
#define PGB_V2(NT, MB, TW, TH)                                                                    \
  V2Inst{NT, MB, TW, TH, (const void *)k_fused2<true, NT, MB, TW, TH>,                             \
         (const void *)k_fused2<false, NT, MB, TW, TH>, fused2_smem<NT, TW, TH>(true),             \
         fused2_smem<NT, TW, TH>(false), true}
// the warp-specialised form: sixteen warps of 128 registers
#define PGB_V3(NT, MB, TW, TH)                                                                    \
  V2Inst{NT, MB, TW, TH, (const void *)k_fused3<true, NT, MB, TW, TH>,                             \
         (const void *)k_fused3<false, NT, MB, TW, TH>, fused3_smem<NT, TW, TH>(true),             \
         fused3_smem<NT, TW, TH>(false), false}
const V2Inst kV2[] = {PGB_V2(256, 1, 24, 7), PGB_V2(256, 1, 30, 6), PGB_V2(128, 2, 14, 6), PGB_V3(512, 1, 14, 8),
                      PGB_V3(512, 1, 16, 7)};
#undef PGB_V2
#undef PGB_V3
constexpr int kNV2 = sizeof(kV2) / sizeof(kV2[0]);

// the uniform kernel's default tile: i and j cut evenly in pieces the layout holds
void default_tile2(HostBlock &B, const V2Inst &v) {
  const int pi = (B.nx + v.tw - 1) / v.tw;
  const int pj = (B.ny + v.th - 1) / v.th;
  B.tw = (B.nx + pi - 1) / pi;
  B.th = (B.ny + pj - 1) / pj;
  B.kchunk = (B.nz + 2) / 3;
}

bool tile_fits(const pgb_case *c, int tw, int th) {
  if (!c->use_v2) return tw * th <= FUSED_THREADS;
  return tw <= kV2[c->v2].tw && th <= kV2[c->v2].th;
}

int build_tiles(pgb_case *c) {
  std::vector<TileDev> tiles;
  size_t smem = 0;
  const bool visc = c->phys.simulator == PGB_NAVIER_STOKES;
  for (int b = 0; b < (int)c->blocks.size(); b++) {
    HostBlock &B = c->blocks[b];
    if (B.tw <= 0 || !tile_fits(c, B.tw, B.th)) {
      if (c->use_v2) default_tile2(B, kV2[c->v2]);
      else default_tile(B);
    }
    const size_t need = !c->use_v2 ? fused_smem(B.tw, B.th, visc) : visc ? kV2[c->v2].smvisc : kV2[c->v2].smeuler;
    smem = std::max(smem, need);
    for (int k0 = 0; k0 < B.nz; k0 += B.kchunk)
      for (int j0 = 0; j0 < B.ny; j0 += B.th)
        for (int i0 = 0; i0 < B.nx; i0 += B.tw) {
          TileDev t;
          t.blk = b;
          t.i0 = (short)i0, t.j0 = (short)j0;
          t.tw = (short)std::min(B.tw, B.nx - i0);
          t.th = (short)std::min(B.th, B.ny - j0);
          t.k0 = (short)k0, t.k1 = (short)std::min(B.nz, k0 + B.kchunk);
          tiles.push_back(t);
        }
  }
  // largest first, so the queue's tail is the small tiles
  std::stable_sort(tiles.begin(), tiles.end(), [](const TileDev &x, const TileDev &y) {
    return (long)x.tw * x.th * (x.k1 - x.k0) > (long)y.tw * y.th * (y.k1 - y.k0);
  });
  if (smem > 227 * 1024) return fail(PGB_ERR_ARG, "tile needs more shared memory than a CTA has");
  if (c->d_tiles) cudaFree(c->d_tiles);
  c->d_tiles = nullptr;
  CK(cudaMalloc(&c->d_tiles, sizeof(TileDev) * std::max<size_t>(1, tiles.size())));
  CK(cudaMemcpy(c->d_tiles, tiles.data(), sizeof(TileDev) * tiles.size(), cudaMemcpyHostToDevice));
  c->ntiles = (int)tiles.size();
  c->fused_smem = smem;
  c->tiles_dirty = false;
  for (auto &g : c->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  return PGB_OK;
}

// Each block's uniform form when its metrics allow it: every area vector along
// its axis alone and equal, the inverse Jacobian diagonal and equal, the cell
// centres evenly spaced; the representative values are the block's own.
int detect_uniform(pgb_case *c, bool allow) {
  const int nb = (int)c->blocks.size();
  std::vector<double> h;
  for (int b = 0; b < nb; b++) {
    HostBlock &HB = c->blocks[b];
    BlockDev &D = HB.dev;
    D.uniform = 0;
    if (!allow) continue;
    bool ok = true;
    for (int m = 0; m < PGB_NMETRICS; m++) ok = ok && HB.metrics_set[m];
    if (!ok) continue;
    h.resize((size_t)M_NCOMP * D.vol);
    CK(cudaMemcpy(h.data(), c->d_met + (long long)M_NCOMP * D.cv, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
    auto at = [&](int comp, int i, int j, int k) { return h[(size_t)comp * D.vol + cell_index(D, i + NG, j + NG, k + NG)]; };
    const int n[3] = {D.nx, D.ny, D.nz};
    auto close = [](double x, double ref, double tol) { return std::fabs(x - ref) <= tol * std::fabs(ref); };
    double S[3], Jd[3], ex[3], xL[3], xR[3];
    const double dJ = at(M_DETJINV, 0, 0, 0);
    for (int a = 0; a < 3; a++) {
      S[a] = at(M_S + 3 * a + a, 0, 0, 0);
      Jd[a] = at(M_JINV + 4 * a, 0, 0, 0);
      int o[3] = {0, 0, 0};
      o[a] = -1;
      ex[a] = at(M_XCC + a, 0, 0, 0) - at(M_XCC + a, o[0], o[1], o[2]);
      xL[a] = at(M_XF + 3 * a + a, 0, 0, 0) - at(M_XCC + a, o[0], o[1], o[2]);
      xR[a] = at(M_XF + 3 * a + a, 0, 0, 0) - at(M_XCC + a, 0, 0, 0);
    }
    // every interior cell and its faces; the inverse Jacobian on the first halo layer too
    for (int k = -1; k <= n[2] && ok; k++)
      for (int j = -1; j <= n[1] && ok; j++)
        for (int i = -1; i <= n[0] && ok; i++) {
          const int out = (i < 0 || i >= n[0]) + (j < 0 || j >= n[1]) + (k < 0 || k >= n[2]);
          if (out > 1) continue;
          for (int a = 0; a < 3 && ok; a++)
            for (int e = 0; e < 3; e++) {
              const double J = at(M_JINV + 3 * a + e, i, j, k);
              ok = ok && (a == e ? close(J, Jd[a], 1e-12) : J == 0.0);
            }
          if (out) continue;
          ok = ok && close(at(M_DETJINV, i, j, k), dJ, 1e-12);
          for (int a = 0; a < 3 && ok; a++) {
            int o[3] = {0, 0, 0};
            o[a] = -1;
            for (int e = 0; e < 3; e++) {
              const double s = at(M_S + 3 * a + e, i, j, k);
              ok = ok && (a == e ? close(s, S[a], 1e-12) : s == 0.0);
              const double d = at(M_XCC + e, i, j, k) - at(M_XCC + e, i + o[0], j + o[1], k + o[2]);
              ok = ok && (a == e ? close(d, ex[a], 1e-9) : std::fabs(d) <= 1e-12 * std::fabs(ex[a]));
            }
          }
        }
    if (!ok) continue;
    D.uniform = 1;
    D.detJinv = dJ;
    for (int a = 0; a < 3; a++) {
      D.S[a] = S[a], D.Jd[a] = Jd[a], D.ex[a] = ex[a], D.xL[a] = xL[a], D.xR[a] = xR[a];
      // alpha-damping.mako:13-25 on an area vector along axis a
      const double Sabs = std::sqrt(S[a] * S[a]), Sinv = 1.0 / Sabs;
      const double nrm = S[a] * Sinv;
      const double en = ex[a] * nrm;
      const double dampinv = c->phys.alpha / std::sqrt(en * en);
      D.damp[a] = dampinv * nrm;
    }
  }
  std::vector<BlockDev> devs;
  for (auto &B : c->blocks) devs.push_back(B.dev);
  CK(cudaMemcpy(c->d_blks, devs.data(), sizeof(BlockDev) * devs.size(), cudaMemcpyHostToDevice));
  c->uniform_done = true;
  return PGB_OK;
}

// The fused path's physical registers: a stage may not write the register its
// stencil reads, so such a write goes to a free buffer and the mapping moves;
// a pure write goes back to the register's own buffer when that is free.
// Stepping from the identity mapping, the mappings fall into a cycle; the
// case starts on the cycle (its buffers are still empty then) and the plan is
// the cycle's steps, `period` of them.  A store is dropped when the register's
// next access, going round the stages, is a pure write.
int plan_step(pgb_case *c, std::vector<int> &map, std::vector<FusedStagePlan> &plan) {
  const int nr = c->phys.nregs;
  const int ns = (int)c->stages.size();
  const int dq = c->stages[0].dq;
  auto reads_of = [&](const pgb_combine &cb, int r) {
    if (cb.own && cb.out == r) return true;
    for (int n = 0; n < cb.nterms; n++)
      if (cb.reg[n] == r) return true;
    return false;
  };
  auto live = [&](int s, int r) {
    for (int q = 1; q <= ns; q++) {
      const pgb_stage &st = c->stages[(s + q) % ns];
      if (st.q == r) return true;
      for (int mm = 0; mm < st.ncombine; mm++) {
        if (reads_of(st.combine[mm], r)) return true;
        if (st.combine[mm].out == r) return false;
      }
    }
    return true;
  };
  plan.clear();
  for (int s = 0; s < ns; s++) {
    const pgb_stage &st = c->stages[s];
    FusedStagePlan p{};
    p.qin = map[st.q];
    p.dqbuf = map[dq];
    p.ncomb = st.ncombine;
    int written0 = -1;
    for (int m = 0; m < st.ncombine; m++) {
      const pgb_combine &cb = st.combine[m];
      FusedCombine &f = p.comb[m];
      f.step = cb.step;
      f.nterms = 0;
      if (cb.own) f.src[f.nterms] = cb.out == written0 ? -2 : map[cb.out], f.w[f.nterms++] = cb.wout;
      for (int n = 0; n < cb.nterms; n++) {
        const int r = cb.reg[n];
        f.src[f.nterms] = (r == -1 || r == dq) ? -1 : (r == written0 ? -2 : map[r]);
        f.w[f.nterms++] = cb.w[n];
      }
      auto in_use = [&](int buf) {
        for (int r = 0; r < nr; r++)
          if (r != cb.out && r != dq && map[r] == buf) return true;
        return buf == p.qin;
      };
      int dst;
      if (!cb.own && !in_use(c->canonical[cb.out])) {
        dst = c->canonical[cb.out];
      } else if (map[cb.out] != p.qin) {
        dst = map[cb.out];
      } else {
        dst = -1;
        for (int buf = 0; buf < nr; buf++)
          if (!in_use(buf) && buf != map[cb.out]) {
            dst = buf;
            break;
          }
        if (dst < 0) return fail(PGB_ERR_STATE, "no free register for a stage's output");
      }
      f.out = dst;
      f.write = live(s, cb.out) ? 1 : 0;
      map[cb.out] = dst;
      if (m == 0) written0 = cb.out;
    }
    // dQ's logical register names the one buffer no other register holds
    for (int buf = 0; buf < nr; buf++) {
      bool used = false;
      for (int r = 0; r < nr; r++)
        if (r != dq && map[r] == buf) used = true;
      if (!used) map[dq] = buf;
    }
    plan.push_back(p);
  }
  return PGB_OK;
}

int build_plans(pgb_case *c) {
  const int nr = c->phys.nregs;
  if (c->stages.empty()) return fail(PGB_ERR_STATE, "no stages set");
  c->canonical.resize(nr);
  for (int r = 0; r < nr; r++) c->canonical[r] = r;
  std::vector<std::vector<int>> states{c->canonical};
  std::vector<std::vector<FusedStagePlan>> plans;
  for (int t = 0; t < 8; t++) {
    std::vector<int> map = states.back();
    std::vector<FusedStagePlan> plan;
    RET(plan_step(c, map, plan));
    plans.push_back(plan);
    for (int s = 0; s <= t; s++) {
      if (states[s] != map) continue;
      // steps s .. t repeat
      c->period = t + 1 - s;
      c->plans.assign(plans.begin() + s, plans.end());
      c->maps.assign(states.begin() + s, states.end());
      c->phase = 0;
      c->phys_of = c->maps[0];
      return PGB_OK;
    }
    states.push_back(map);
  }
  return fail(PGB_ERR_STATE, "the register plan does not repeat within eight steps");
}

int grid_for(long long n, int threads) { return (int)std::max<long long>(1, (n + threads - 1) / threads); }

enum { K_HALO = 0, K_FUSED = 1, K_BLOCK = 2, K_COMBINE = 3 };

// after every launch: count it, and under pgb_step_timed record an event
void mark(pgb_case *c, int kind, int &count) {
  count++;
  if (!c->timing) return;
  if (c->tnext >= c->tev.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->tev.push_back(e);
  }
  cudaEventRecord(c->tev[c->tnext++], c->stream);
  c->tkind.push_back(kind);
}

// Whether every face of every block lets a stage read across it from the
// neighbour's cells in place of its halo: joined to a neighbour low face to
// high face in the identity orientation, unrotated, with both blocks at least
// NG cells thick along the axis, so a halo cell's source lies one face away
// along each axis it is outside (what locate finds, axis by axis).
bool faces_pullable(const pgb_case *c) {
  for (const HostBlock &B : c->blocks) {
    const int n[3] = {B.nx, B.ny, B.nz};
    for (int f = 0; f < 6; f++) {
      const int a = f / 2, nb = B.nbr[f];
      if (nb < 0 || B.rot[f] || B.bc[f] >= 0 || n[a] < NG) return false;
      if (B.nbrface[f] != (f % 2 ? f : f + 2)) return false;
      for (int d = 0; d < 3; d++)
        if (B.orient[f][d] != d + 1) return false;
      const HostBlock &N = c->blocks[nb];
      const int m[3] = {N.nx, N.ny, N.nz};
      if (m[a] < NG) return false;
      for (int d = 0; d < 3; d++)
        if (d != a && m[d] != n[d]) return false;
    }
  }
  return true;
}

// whether the case's uniform stages pull across faces: wanted, the faces
// allow it, the instance reads that way, and no face's halo comes from an
// exchange with another case
bool pulls(const pgb_case *c) {
  return c->pull_want && c->pull_faces && c->use_v2 && c->v2 >= 0 && c->v2 < kNV2 && kV2[c->v2].pull &&
         c->nxrecv == 0;
}

// the uniform kernel of the case's instance
const void *v2_kernel(const pgb_case *c) {
  if (c->v2 < 0 || c->v2 >= kNV2) return nullptr;
  return c->phys.simulator == PGB_NAVIER_STOKES ? kV2[c->v2].fvisc : kV2[c->v2].feuler;
}

// one stage of the fused path; dtp, when given, the step size the combines read
// in place of the case's
int launch_fused(pgb_case *c, const FusedStagePlan &p, int stage_index, int &count, const double *dtp = nullptr) {
  FusedArgs a{};
  a.blks = c->d_blks;
  a.tiles = c->d_tiles;
  a.ntiles = c->ntiles;
  a.counter = c->d_counter + stage_index;
  a.met = c->d_met;
  for (int r = 0; r < c->phys.nregs; r++) a.R[r] = c->d_reg[r];
  a.qin = p.qin;
  a.ncomb = p.ncomb;
  a.comb[0] = p.comb[0];
  a.comb[1] = p.comb[1];
  // the registers the combines read, as slots the uniform kernel fills ahead
  a.npre = 0;
  for (int m = 0; m < p.ncomb; m++) {
    a.combp[m] = p.comb[m];
    for (int n = 0; n < p.comb[m].nterms; n++) {
      const int r = p.comb[m].src[n];
      if (r < 0) continue;
      int slot = -1;
      for (int q = 0; q < a.npre; q++)
        if (a.pre[q] == r) slot = q;
      if (slot < 0) {
        if (a.npre == 3) return fail(PGB_ERR_STATE, "a stage reads more than three registers");
        slot = a.npre;
        a.pre[a.npre++] = r;
      }
      a.combp[m].src[n] = slot;
    }
  }
  // the fixed form: each combine's terms onto (p0, p1, dt dQ, out0), in order
  for (int m = 0; m < 2; m++) {
    for (int q = 0; q < 4; q++) a.cw[m][q] = 0.0;
    a.outp[m] = nullptr;
    a.write[m] = 0;
  }
  for (int m = 0; m < p.ncomb; m++) {
    const FusedCombine &cb = a.combp[m];
    int last = -1;
    for (int n = 0; n < cb.nterms; n++) {
      const int sidx = cb.src[n];
      const int q = sidx == -1 ? 2 : sidx == -2 ? 3 : sidx;
      // the form sums p0, p1, dQ, out0 in that order: a combine whose terms
      // come in another order, or that reads a slot twice, has no fixed form
      if (q <= last || (q == 3 && m == 0) || (q == 2 && !(cb.step && n == cb.nterms - 1)))
        return fail(PGB_ERR_STATE, "a stage whose combines the uniform kernel's fixed form does not take");
      if (q < 2 && cb.step && n == cb.nterms - 1)
        return fail(PGB_ERR_STATE, "a stage whose dt falls on a register the fixed form does not scale");
      last = q;
      a.cw[m][q] = cb.w[n];
    }
    a.outp[m] = c->d_reg[cb.out];
    a.write[m] = cb.write;
  }
  for (int q = 0; q < 2; q++) a.prep[q] = q < a.npre ? c->d_reg[a.pre[q]] : nullptr;
  a.dt = dtp ? dtp : c->d_dt;
  // the stencil register's halo first, unless the stage reads across faces
  a.pull = pulls(c) ? 1 : 0;
  a.nbr27 = c->d_nbr27;
  if (!a.pull) {
    halo_fill_case(c, c->d_reg[p.qin], c->ne, 1);
    mark(c, K_HALO, count);
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool any_general = !c->use_v2;
  const bool visc = c->phys.simulator == PGB_NAVIER_STOKES;
  const size_t sm = c->fused_smem;
  if (c->use_v2) {
    if (a.npre > 2) return fail(PGB_ERR_STATE, "the uniform kernels stage at most two registers a stage reads");
    const int grid = std::min(c->ntiles, sms * c->v2_ctas);
    const void *fn = v2_kernel(c);
    if (!fn) return fail(PGB_ERR_ARG, "no uniform kernel of that shape");
    void *args[] = {&a};
    CK(cudaLaunchKernel(fn, dim3(grid), dim3(kV2[c->v2].nt), args, sm, c->stream));
    mark(c, K_FUSED, count);
    return PGB_OK;
  }
  const int grid = std::min(c->ntiles, sms * 2);
  if (visc) {
    if (any_general) k_fused1<true, false><<<grid, FUSED_THREADS, sm, c->stream>>>(a);
    else k_fused1<true, true><<<grid, FUSED_THREADS, sm, c->stream>>>(a);
  } else {
    if (any_general) k_fused1<false, false><<<grid, FUSED_THREADS, sm, c->stream>>>(a);
    else k_fused1<false, true><<<grid, FUSED_THREADS, sm, c->stream>>>(a);
  }
  mark(c, K_FUSED, count);
  CK(cudaGetLastError());
  return PGB_OK;
}

int fused_attrs(pgb_case *c) {
  const int sm = (int)c->fused_smem;
  if (c->use_v2) {
    const void *fn = v2_kernel(c);
    if (!fn) return fail(PGB_ERR_ARG, "no uniform kernel of that shape");
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    int n = 1;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kV2[c->v2].nt, c->fused_smem));
    c->v2_ctas = std::max(1, n);
    return PGB_OK;
  }
  CK(cudaFuncSetAttribute(k_fused1<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_fused1<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_fused1<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_fused1<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  return PGB_OK;
}

// one step of the fused path at the current phase
PlainCase plain_case(pgb_case *c, std::vector<BlockDev> &hb);
int prestep_plain(pgb_case *c, int qphys, int &count, int first);
struct MarkCtx {
  pgb_case *c;
  int *count;
};
void mark_cb(void *ctx, int kind);

// the CFL reduction of physical register qphys into d_cfl
int cfl_pass(pgb_case *c, int qphys, int &count);

// under the cfl controller a step opens with the reduction of its start
// register and the step size it gives (peregrine/multiblock/solver.py:366-370)
int cfl_prologue(pgb_case *c, int qphys, int &count) {
  if (!c->ctrl_cfl) return PGB_OK;
  RET(cfl_pass(c, qphys, count));
  k_cfldt<<<1, 1, 0, c->stream>>>(c->d_dt, c->d_cfl, c->d_ctrl);
  mark(c, K_COMBINE, count);
  return PGB_OK;
}

// one stage of the fused passes (react.cuh): the plan's combines on physical
// registers; with dq set (a right-hand side alone) no combine, dQ stored there
int launch_react(pgb_case *c, const FusedStagePlan &p, int &count, int dq = -1) {
  RStage r{};
  r.Q = c->d_reg[p.qin];
  r.dQ = c->d_reg[dq >= 0 ? dq : p.dqbuf];
  r.write_dq = dq >= 0;
  r.ncomb = dq >= 0 ? 0 : p.ncomb;
  for (int m = 0; m < r.ncomb; m++) {
    const FusedCombine &f = p.comb[m];
    RCombine &rc = r.comb[m];
    rc.out = c->d_reg[f.out];
    rc.nterms = f.nterms, rc.step = f.step, rc.write = f.write;
    for (int n = 0; n < f.nterms; n++) {
      rc.src[n] = f.src[n] < 0 ? f.src[n] : 0;
      rc.X[n] = f.src[n] >= 0 ? c->d_reg[f.src[n]] : nullptr;
      rc.w[n] = f.w[n];
    }
  }
  std::vector<BlockDev> hb;
  PlainCase pc = plain_case(c, hb);
  MarkCtx mc{c, &count};
  pc.mark = mark_cb;
  pc.ctx = &mc;
  pc.packed = 1;
  c->state_stale = false;
  return kPlain[c->phys.ns - 1].fused(&pc, &r);
}

int step_fused(pgb_case *c, int &count) {
  const auto &plan = c->plans[c->phase];
  if (c->form != 2) c->state_stale = true;
  RET(cfl_prologue(c, plan[0].qin, count));
  if (c->form == 2 && sim_df(c->phys.simulator)) {
    // the double flux's step start, each pass one launch over every block
    struct Packed {
      pgb_case *c;
      bool was;
      ~Packed() { c->packed = was; }
    } keep{c, c->packed};
    c->packed = true;
    RET(prestep_plain(c, plan[0].qin, count, 0));
  }
  CK(cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned int) * plan.size(), c->stream));
  for (int s = 0; s < (int)plan.size(); s++)
    RET(c->form == 2 ? launch_react(c, plan[s], count) : launch_fused(c, plan[s], s, count));
  if (c->ctrl_cfl) {
    k_clock<<<1, 1, 0, c->stream>>>(c->d_clock, c->d_dt);
    mark(c, K_COMBINE, count);
  }
  c->phase = (c->phase + 1) % c->period;
  c->phys_of = c->maps[c->phase];
  return PGB_OK;
}

// The right-hand side alone on the fused path: the stage kernel with one
// combine, out = 1 x dt x dQ at dt = 1 (no register term, the fixed form's
// other weights zero), so it writes exactly the dQ it forms.  The halo fill
// of q comes first, as in a stage.
int rhs_fused(pgb_case *c, int qphys, int dqphys, int &count) {
  if (c->form == 2) {
    FusedStagePlan p{};
    p.qin = qphys;
    return launch_react(c, p, count, dqphys);
  }
  FusedStagePlan p{};
  p.qin = qphys;
  p.ncomb = 1;
  FusedCombine &f = p.comb[0];
  f.step = 1;
  f.nterms = 1;
  f.src[0] = -1;
  f.w[0] = 1.0;
  f.out = dqphys;
  f.write = 1;
  c->state_stale = true;
  CK(cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned int), c->stream));
  return launch_fused(c, p, 0, count, c->d_one);
}

// the per-cell state, kept between right-hand sides: an iterative eos starts
// from each cell's last T
int ensure_state(pgb_case *c) {
  if (c->d_state) return PGB_OK;
  const size_t n = (size_t)c->cells;
  CK(cudaMalloc(&c->d_state, sizeof(double) * SW * n));
  CK(cudaMemsetAsync(c->d_state, 0, sizeof(double) * SW * n, c->stream));
  return PGB_OK;
}

int ensure_scratch(pgb_case *c) {
  RET(ensure_state(c));
  if (c->d_tr) return PGB_OK;
  const int ns = c->phys.ns, ne = c->ne, ngrad = ne - 1;
  const size_t n = (size_t)c->cells;
  CK(cudaMalloc(&c->d_tr, sizeof(double) * (2 + ns) * n));
  CK(cudaMalloc(&c->d_hsp, sizeof(double) * ns * n));
  CK(cudaMalloc(&c->d_grads, sizeof(double) * 3 * ngrad * n));
  // the double flux writes its energy row twice: one row more per face
  const int nf = ne + sim_df(c->phys.simulator);
  for (int a = 0; a < 3; a++) CK(cudaMalloc(&c->d_F[a], sizeof(double) * nf * n));
  CK(cudaMemsetAsync(c->d_tr, 0, sizeof(double) * (2 + ns) * n, c->stream));
  CK(cudaMemsetAsync(c->d_hsp, 0, sizeof(double) * ns * n, c->stream));
  CK(cudaMemsetAsync(c->d_grads, 0, sizeof(double) * 3 * ngrad * n, c->stream));
  for (int a = 0; a < 3; a++) CK(cudaMemsetAsync(c->d_F[a], 0, sizeof(double) * nf * n, c->stream));
  if (c->phys.chemistry == PGB_CHEM_SUBSTEPPED) {
    // a bin's segment holds every interior cell, so it never fills
    CK(cudaMalloc(&c->d_subs, sizeof(int) * n));
    CK(cudaMemsetAsync(c->d_subs, 0, sizeof(int) * n, c->stream));
    CK(cudaMalloc(&c->d_stiffhead, sizeof(unsigned int) * (16 + 2)));
    CK(cudaMemsetAsync(c->d_stiffhead, 0, sizeof(unsigned int) * (16 + 2), c->stream));
    CK(cudaMalloc(&c->d_stiffcells, sizeof(int2) * (size_t)c->subopt.bins * (size_t)c->interior_cells));
  }
  return PGB_OK;
}

void mark_cb(void *ctx, int kind) {
  MarkCtx *m = (MarkCtx *)ctx;
  mark(m->c, kind, *m->count);
}

PlainCase plain_case(pgb_case *c, std::vector<BlockDev> &hb) {
  hb.clear();
  for (auto &B : c->blocks) hb.push_back(B.dev);
  PlainCase pc{};
  pc.d_blks = c->d_blks;
  pc.h_blks = hb.data();
  pc.nblocks = (int)hb.size();
  pc.state = c->d_state, pc.tr = c->d_tr, pc.hsp = c->d_hsp, pc.grads = c->d_grads;
  for (int a = 0; a < 3; a++) pc.F[a] = c->d_F[a];
  pc.met = c->d_met;
  pc.halo = c->d_halo;
  pc.nhalo = c->nhalo, pc.nhalo_l0 = c->nhalo_l0;
  pc.boxes = c->d_boxes, pc.boxcta = c->d_boxcta, pc.nboxcta = c->nboxcta;
  pc.boxrest = c->d_boxrest, pc.nboxrest = c->nboxrest;
  pc.rots = c->d_rots;
  pc.visc = sim_visc(c->phys.simulator);
  pc.packed = c->packed ? 1 : 0;
  pc.primary = c->phys.primary, pc.recon = c->phys.recon, pc.limiter = c->phys.limiter;
  pc.chem = c->phys.chemistry;
  pc.subopt = c->subopt;
  pc.subs = c->d_subs;
  pc.stiff = StiffList{c->d_stiffhead, c->d_stiffcells, c->interior_cells};
  pc.df = sim_df(c->phys.simulator);
  pc.realgas = c->phys.eos == PGB_EOS_REALGAS || c->phys.eos == PGB_EOS_REALGAS_DF;
  pc.bchalo = c->d_bcface[0], pc.bcgrad = c->d_bcface[1], pc.bcwall = c->d_bcface[2];
  pc.nbchalo = c->nbcface[0], pc.nbcgrad = c->nbcface[1], pc.nbcwall = c->nbcface[2];
  pc.bchalo_n = c->bcthreads[0], pc.bcgrad_n = c->bcthreads[1], pc.bcwall_n = c->bcthreads[2];
  pc.bcent = c->d_bcent, pc.bcops = c->d_bcops;
  pc.clock = c->d_clock, pc.dt = c->d_dt;
  pc.gensrc = c->gen_src, pc.genmath = c->d_math, pc.blkstride = (int)sizeof(BlockDev);
  // blocks whose halo is a large share of their cells take the interior cell
  // pass, where the case's own halo table fills every halo cell (a shard's
  // traded halo cells get Q alone, so their fields are formed in place)
  pc.rcell_inner = c->nxrecv == 0 && c->cells > (long long)(1.3 * (double)c->interior_cells) ? 1 : 0;
  pc.tfrac = 0.0;
  pc.stream = c->stream;
  return pc;
}

// the double flux's freeze on register qphys: at every step's start off the
// frozen planes (first 0), or once after the state was set, off the eos
// (first 1; the reference's initialize graph,
// peregrine/simulator/eulerdf/simulator.py:63-66)
int prestep_plain(pgb_case *c, int qphys, int &count, int first) {
  if (!sim_df(c->phys.simulator)) return PGB_OK;
  RET(ensure_scratch(c));
  std::vector<BlockDev> hb;
  PlainCase pc = plain_case(c, hb);
  MarkCtx mc{c, &count};
  pc.mark = mark_cb;
  pc.ctx = &mc;
  RET(kPlain[c->phys.ns - 1].prestep(&pc, c->d_reg[qphys], first));
  if (first) c->df_fresh = false;
  return PGB_OK;
}

// the double flux's planes for a state just set
int df_settle(pgb_case *c, int qphys) {
  if (!sim_df(c->phys.simulator) || !c->df_fresh) return PGB_OK;
  int count = 0;
  return prestep_plain(c, qphys, count, 1);
}

int rhs_plain(pgb_case *c, int qphys, int dqphys, int &count, double tfrac = 0.0) {
  RET(ensure_scratch(c));
  std::vector<BlockDev> hb;
  PlainCase pc = plain_case(c, hb);
  MarkCtx mc{c, &count};
  pc.mark = mark_cb;
  pc.ctx = &mc;
  pc.tfrac = tfrac;
  c->state_stale = false;
  return kPlain[c->phys.ns - 1].rhs(&pc, c->d_reg[qphys], c->d_reg[dqphys]);
}

int cfl_pass(pgb_case *c, int qphys, int &count) {
  CK(cudaMemsetAsync(c->d_cfl, 0, sizeof(double) * 3, c->stream));
  std::vector<BlockDev> hb;
  PlainCase pc = plain_case(c, hb);
  MarkCtx mc{c, &count};
  pc.mark = mark_cb;
  pc.ctx = &mc;
  return kPlain[c->phys.ns - 1].cflmax(&pc, c->d_reg[qphys], c->d_cfl);
}

// a stage's combines on the registers as they are (the reference's advance
// graph, peregrine/integrators/rungekutta.py:21-26)
void combine_stage(pgb_case *c, const pgb_stage &st, int &count) {
  const int TH = 256;
  const auto &map = c->phys_of;
  for (int m = 0; m < st.ncombine; m++) {
      const pgb_combine &cb = st.combine[m];
      CombineDev cd{};
      cd.out = c->d_reg[map[cb.out]];
      cd.own = cb.own;
      cd.wout = cb.wout;
      cd.nterms = cb.nterms;
      cd.step = cb.step;
      for (int n = 0; n < cb.nterms; n++) {
        const int r = cb.reg[n] < 0 ? st.dq : cb.reg[n];
        cd.X[n] = c->d_reg[map[r]];
        cd.w[n] = cb.w[n];
      }
      if (c->packed) {
        // one launch over every block, a grid row each
        long long most = 0;
        for (const HostBlock &B : c->blocks) most = std::max(most, (long long)B.nx * B.ny * B.nz);
        k_combine<<<dim3(grid_for(most, TH), (unsigned)c->blocks.size(), 1), TH, 0, c->stream>>>(c->d_blks, 0, c->ne,
                                                                                                 cd, c->d_dt);
        mark(c, K_COMBINE, count);
        continue;
      }
      for (int b = 0; b < (int)c->blocks.size(); b++) {
        const BlockDev &D = c->blocks[b].dev;
        k_combine<<<grid_for((long long)D.nx * D.ny * D.nz, TH), TH, 0, c->stream>>>(c->d_blks, b, c->ne, cd, c->d_dt);
        mark(c, K_COMBINE, count);
      }
  }
}

int step_plain(pgb_case *c, int &count) {
  const auto &map = c->phys_of;
  if (!c->stages.empty()) RET(cfl_prologue(c, map[c->stages[0].q], count));
  if (!c->stages.empty()) RET(prestep_plain(c, map[c->stages[0].q], count, 0));
  for (const pgb_stage &st : c->stages) {
    RET(rhs_plain(c, map[st.q], map[st.dq], count, st.tfrac));
    combine_stage(c, st, count);
  }
  // the clock moves on by dt where boundaries read it or the step size is the device's
  if (c->nbcface[0] || c->ctrl_cfl) {
    k_clock<<<1, 1, 0, c->stream>>>(c->d_clock, c->d_dt);
    mark(c, K_COMBINE, count);
  }
  CK(cudaGetLastError());
  return PGB_OK;
}

// the boundary passes' face tables: every boundary face given an entry in the
// halo pass, the inflows' and outflows' faces again in the gradient pass when
// the case is viscous, the walls' in the wall pass; each table's threads end
// to end, closed by a sentinel holding the pass's thread count
int build_bcs(pgb_case *c) {
  std::vector<BcFace> t[3];
  long long n[3] = {0, 0, 0};
  const bool visc = sim_visc(c->phys.simulator);
  for (int b = 0; b < (int)c->blocks.size(); b++) {
    const HostBlock &B = c->blocks[b];
    const int ext[3] = {B.nx, B.ny, B.nz};
    for (int f = 0; f < 6; f++) {
      const int e = B.bc[f];
      if (e < 0) continue;
      const int a = f / 2;
      const long long plane = (long long)ext[a == 0 ? 1 : 0] * ext[a == 2 ? 1 : 2];
      const bool wall = bc_is_wall(c->bc_entries[e].kind);
      t[0].push_back(BcFace{b, f, e, 0, n[0]});
      n[0] += NG * plane;
      if (visc && !wall) {
        t[1].push_back(BcFace{b, f, e, 0, n[1]});
        n[1] += NG * plane;
      }
      if (wall) {
        t[2].push_back(BcFace{b, f, e, 0, n[2]});
        n[2] += plane;
      }
    }
  }
  for (int p = 0; p < 3; p++) {
    c->nbcface[p] = (int)t[p].size();
    c->bcthreads[p] = n[p];
    if (t[p].empty()) continue;
    t[p].push_back(BcFace{0, 0, 0, 0, n[p]});
    CK(cudaMalloc(&c->d_bcface[p], sizeof(BcFace) * t[p].size()));
    CK(cudaMemcpy(c->d_bcface[p], t[p].data(), sizeof(BcFace) * t[p].size(), cudaMemcpyHostToDevice));
  }
  if (!c->bc_entries.empty()) {
    CK(cudaMalloc(&c->d_bcent, sizeof(BcEntry) * c->bc_entries.size()));
    CK(cudaMemcpy(c->d_bcent, c->bc_entries.data(), sizeof(BcEntry) * c->bc_entries.size(), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_bcops, sizeof(BcOp) * std::max<size_t>(1, c->bc_ops.size())));
    if (!c->bc_ops.empty())
      CK(cudaMemcpy(c->d_bcops, c->bc_ops.data(), sizeof(BcOp) * c->bc_ops.size(), cudaMemcpyHostToDevice));
  }
  return PGB_OK;
}

int prepare(pgb_case *c, bool fused) {
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  RET(set_current(c));
  if (fused) {
    const int form = batched_form(c);
    if (form != c->form) c->tiles_dirty = true;
    c->form = form;
  }
  // the fused passes read the per-block path's state, transport, gradient
  // and face arrays and keep the metric arrays' form
  if (fused && c->form == 2) return ensure_scratch(c);
  // the uniform forms are the batched path's alone: the per-block path reads
  // the metric arrays, so a per-block call leaves the detection to the first
  // batched step
  if (fused && !c->uniform_done) {
    RET(detect_uniform(c, true));
    bool all = true;
    for (auto &B : c->blocks) all = all && B.dev.uniform;
    if (all != c->use_v2) c->tiles_dirty = true;
    c->use_v2 = all;
  }
  if (fused) {
    if (c->tiles_dirty) RET(build_tiles(c));
    RET(fused_attrs(c));
  }
  return PGB_OK;
}

// the generated kernel reads a block record's leading fields by these offsets
static_assert(offsetof(BlockDev, nx) == 0 && offsetof(BlockDev, Z) == 20 && offsetof(BlockDev, vol) == 24 &&
                  offsetof(BlockDev, cv) == 32,
              "the generated source's block record");

// The coupled chemistry's source generated for the case's mechanism and
// compiled for the device (rategen.cu); where NVRTC is missing or the case
// asks for the table-driven kernel, that kernel stays in use
int build_generated(pgb_case *c) {
  c->gen_src = nullptr;
  if (c->phys.chemistry != PGB_CHEM_COUPLED || !c->mech) {
    c->gen_why = "the case has no coupled chemistry";
    return PGB_OK;
  }
  if (!c->gen_want) {
    c->gen_why = "the case asked for the table-driven kernel";
    return PGB_OK;
  }
  std::string cubin;
  if (!rates_compile(rates_source(*c->mech, c->sp, c->phys.ns), cubin, c->gen_why)) return PGB_OK;
  CK(cudaLibraryLoadData(&c->gen_lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  cudaKernel_t k = nullptr;
  CK(cudaLibraryGetKernel(&k, c->gen_lib, "pgb_gen_source"));
  MathTables mt;
  math_tables_fill(mt);
  CK(cudaMalloc(&c->d_math, sizeof(MathTables)));
  CK(cudaMemcpy(c->d_math, &mt, sizeof(MathTables), cudaMemcpyHostToDevice));
  c->gen_src = (const void *)k;
  c->gen_why.clear();
  return PGB_OK;
}

}  // namespace

extern "C" {

const char *pgb_last_error(void) { return g_err.c_str(); }

// sets the error text of pgb_last_error from the library's other files; not
// part of the ABI
__attribute__((visibility("hidden"))) int pgb_internal_fail(int code, const char *msg) { return fail(code, msg); }
int pgb_version(void) { return 1; }

int pgb_device_init(int ordinal) {
  int n = 0;
  CK(cudaGetDeviceCount(&n));
  if (ordinal < 0 || ordinal >= n) return fail(PGB_ERR_ARG, "no such device");
  CK(cudaSetDevice(ordinal));
  CK(cudaFree(nullptr));
  return PGB_OK;
}

int pgb_device_count(int *count) {
  if (!count) return fail(PGB_ERR_ARG, "null count");
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    cudaGetLastError();
  }
  return PGB_OK;
}

int pgb_device_sync(void) {
  CK(cudaDeviceSynchronize());
  return PGB_OK;
}

int pgb_mem_info(size_t *free_bytes, size_t *total_bytes) {
  CK(cudaMemGetInfo(free_bytes, total_bytes));
  return PGB_OK;
}

int pgb_case_create(const pgb_physics *phys, pgb_case **out) {
  if (!phys || !out) return fail(PGB_ERR_ARG, "null argument");
  if (phys->ns < 1 || phys->ns > MAXNS) return fail(PGB_ERR_ARG, "ns out of range");
  if (phys->nregs < 2 || phys->nregs > MAXREGS) return fail(PGB_ERR_ARG, "nregs out of range");
  if (phys->eos < PGB_EOS_CPG || phys->eos > PGB_EOS_REALGAS_DF)
    return fail(PGB_ERR_UNSUPPORTED, "no such eos");
  if (phys->simulator < PGB_EULER || phys->simulator > PGB_NAVIER_STOKES_DF) return fail(PGB_ERR_ARG, "no such simulator");
  if (sim_df(phys->simulator) != (phys->eos == PGB_EOS_REALGAS_DF))
    return fail(PGB_ERR_ARG, "the double flux freezes the real gas's tangent plane: euler-df and navier-stokes-df take "
                             "real-gas-df, and that eos one of them");
  if (phys->primary < PGB_FLUX_KEPAEC || phys->primary > PGB_FLUX_AUSMUP)
    return fail(PGB_ERR_ARG, "no such flux function");
  // the double flux's flux functions (peregrine/simulator/eulerdf/kernels/flux/function/)
  if (sim_df(phys->simulator) && (phys->primary == PGB_FLUX_HLLC || phys->chemistry != PGB_CHEM_NONE))
    return fail(PGB_ERR_UNSUPPORTED, "the double flux takes kepaec, rusanov or ausmup, without chemistry");
  if (phys->recon != PGB_RECON_CONSTANT && phys->recon != PGB_RECON_MUSCL)
    return fail(PGB_ERR_ARG, "no such reconstruction");
  if (phys->recon == PGB_RECON_MUSCL && (phys->limiter < 1 || phys->limiter > 5))
    return fail(PGB_ERR_ARG, "muscl needs a limiter: koren, minmod, mc, superbee or vanleer");
  if (phys->primary == PGB_FLUX_KEPAEC && phys->recon != PGB_RECON_CONSTANT)
    return fail(PGB_ERR_UNSUPPORTED, "kepaec is a two-point flux of the cells as they are; it takes no muscl sides");
  if (sim_visc(phys->simulator) && phys->trans != PGB_TRANS_CONSTANT && phys->trans != PGB_TRANS_KINETIC)
    return fail(PGB_ERR_UNSUPPORTED, "the viscous path takes constant or kinetic-theory transport");
  if (phys->trans == PGB_TRANS_KINETIC && phys->eos == PGB_EOS_CPG)
    return fail(PGB_ERR_ARG, "kinetic-theory transport needs the thermally perfect caloric");
  if (phys->chemistry < PGB_CHEM_NONE || phys->chemistry > PGB_CHEM_SUBSTEPPED)
    return fail(PGB_ERR_UNSUPPORTED, "the chemistry takes none, coupled or sub-stepped");
  if (phys->chemistry != PGB_CHEM_NONE && phys->eos != PGB_EOS_TPG)
    return fail(PGB_ERR_UNSUPPORTED, "finite-rate chemistry takes the thermally perfect gas in this build");
  auto c = std::make_unique<pgb_case>();
  c->uid = ++g_next_uid;
  c->phys = *phys;
  c->ne = 4 + phys->ns;
  // the stream and events are made at finalize: until then a case is host
  // data alone (a partitioner lists a grid's halo on a machine without a GPU)
  *out = c.release();
  return PGB_OK;
}

int pgb_case_destroy(pgb_case *c) {
  if (!c) return PGB_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto &g : c->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto &r : c->d_reg)
    if (r) cudaFree(r);
  void *ptrs[] = {c->d_blks, c->d_met, c->d_dt, c->d_one, c->d_xsend, c->d_xrecv, c->d_xsvol, c->d_xrvol, c->d_halo, c->d_boxes, c->d_boxcta, c->d_boxrest, c->d_state, c->d_tr, c->d_hsp, c->d_grads,
                  c->d_F[0], c->d_F[1], c->d_F[2], c->d_prims, c->d_tiles, c->d_counter, c->d_stage,
                  c->d_bcent, c->d_bcops, c->d_bcface[0], c->d_bcface[1], c->d_bcface[2], c->d_clock,
                  c->d_cfl, c->d_ctrl, c->d_subs, c->d_stiffhead, c->d_stiffcells, c->d_rots, c->d_nbr27};
  if (c->gen_lib) cudaLibraryUnload(c->gen_lib);
  if (c->d_math) cudaFree(c->d_math);
  for (cudaEvent_t e : c->tev) cudaEventDestroy(e);
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) forget_stream(c->stream), cudaStreamDestroy(c->stream);
  delete c;
  return PGB_OK;
}

int pgb_case_set_table(pgb_case *c, const char *name, const double *values, long n) {
  if (!c || !name || (!values && n)) return fail(PGB_ERR_ARG, "null argument");
  if (n < 0) return fail(PGB_ERR_ARG, "negative size");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  c->tables[name] = std::vector<double>(values, values + n);
  return PGB_OK;
}

int pgb_case_set_mechanism(pgb_case *c, const pgb_mechanism *m) {
  if (!c || !m) return fail(PGB_ERR_ARG, "null argument");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  if (c->phys.chemistry == PGB_CHEM_NONE) return fail(PGB_ERR_STATE, "the case has no chemistry");
  const int ns = c->phys.ns;
  if (m->nr < 0 || m->nr > MAXRXN) return fail(PGB_ERR_UNSUPPORTED, "at most 64 reactions in this build");
  if (m->nr && !m->rxn) return fail(PGB_ERR_ARG, "null reactions");
  if (m->ntb < 0 || m->ntb > MAXTB || (m->ntb && !m->tb)) return fail(PGB_ERR_UNSUPPORTED, "at most 8 third-body sets");
  if (m->ntroe < 0 || m->ntroe > MAXTROE || m->nlfc < 0 || m->nlfc > MAXLFC || (m->ntroe && !m->lfcpoly))
    return fail(PGB_ERR_UNSUPPORTED, "at most 8 Troe reactions of 16 fit terms");
  if (m->ng < 1 || m->ng > MAXT + 1 || !m->gpoly) return fail(PGB_ERR_ARG, "the Gibbs fits take 1 to 9 terms");
  if (!(m->maxgain > 0.0)) return fail(PGB_ERR_ARG, "maxgain is positive");
  auto M = std::make_unique<Mech>();
  std::memset(M.get(), 0, sizeof(Mech));
  M->nr = m->nr, M->ntb = m->ntb, M->nlfc = m->nlfc, M->ngp = m->ng;
  M->logprefRu = m->logprefRu, M->prefRu = m->prefRu, M->Rupref = m->Rupref, M->logcfloor = m->logcfloor;
  M->cfloor = std::exp(m->logcfloor);
  M->troeuc = m->troeuc, M->troeuhinv = m->troeuhinv;
  // the fold's clamp and the floor of a Troe centre with no terms, as the
  // reference works them out on the host (finiterate.mako:128-133, 50-52)
  M->expclamp = std::log(DBL_MAX) - std::log(2.0 * m->maxgain);
  M->lfcfloor = std::log(DBL_MIN) * 0.4342944819032518;
  for (int j = 0; j < m->ntb; j++) {
    const pgb_thirdbody &t = m->tb[j];
    if (t.neff < 0 || t.neff > ns) return fail(PGB_ERR_ARG, "a third-body set's efficiencies exceed the species");
    M->tbdefeff[j] = t.defeff;
    M->tbneff[j] = t.neff;
    for (int i = 0; i < t.neff; i++) {
      if (t.effsp[i] < 0 || t.effsp[i] >= ns) return fail(PGB_ERR_ARG, "a third body names no species");
      M->tbeffsp[j][i] = t.effsp[i];
      M->tbeffdev[j][i] = t.effdev[i];
    }
  }
  for (int k = 0; k < m->ntroe; k++)
    for (int t = 0; t < m->nlfc; t++) M->lfcpoly[k][t] = m->lfcpoly[k * m->nlfc + t];
  for (int n = 0; n < ns; n++)
    for (int t = 0; t < m->ng; t++) M->gpoly[n][t] = m->gpoly[n * m->ng + t];
  bool logform = false, product = false;
  for (int k = 0; k < m->nr; k++) {
    const pgb_reaction &r = m->rxn[k];
    Rxn &d = M->rxn[k];
    if (r.kind < PGB_RXN_ELEMENTARY || r.kind > PGB_RXN_TROE) return fail(PGB_ERR_ARG, "no such reaction kind");
    if ((r.kind != PGB_RXN_ELEMENTARY) && (r.tb < 0 || r.tb >= m->ntb))
      return fail(PGB_ERR_ARG, "a third-body reaction names no set");
    if (r.kind == PGB_RXN_TROE && r.nfcent > 0 && (r.troe < 0 || r.troe >= m->ntroe || m->nlfc < 1))
      return fail(PGB_ERR_ARG, "a Troe reaction names no fit");
    if (r.nfwd < 0 || r.nfwd > PGB_MAXSIDE || r.nreact < 0 || r.nreact > PGB_MAXSIDE || r.nprod < 0 ||
        r.nprod > PGB_MAXSIDE || r.nnet < 0 || r.nnet > PGB_MAXNET)
      return fail(PGB_ERR_UNSUPPORTED, "a reaction's side is longer than this build takes");
    d.kind = r.kind, d.reversible = r.reversible, d.product = r.product, d.tb = r.tb, d.troe = r.troe;
    d.nfcent = r.nfcent, d.nfwd = r.nfwd, d.nreact = r.nreact, d.nprod = r.nprod, d.nnet = r.nnet;
    auto sp_ok = [&](int sp) { return sp >= 0 && sp < ns; };
    for (int j = 0; j < r.nfwd; j++) {
      if (!sp_ok(r.fwdsp[j])) return fail(PGB_ERR_ARG, "a reaction names no species");
      d.fwdsp[j] = r.fwdsp[j], d.fwdorder[j] = r.fwdorder[j];
    }
    for (int j = 0; j < r.nreact; j++) {
      if (!sp_ok(r.reactsp[j])) return fail(PGB_ERR_ARG, "a reaction names no species");
      d.reactsp[j] = r.reactsp[j], d.reactnu[j] = r.reactnu[j];
    }
    for (int j = 0; j < r.nprod; j++) {
      if (!sp_ok(r.prodsp[j])) return fail(PGB_ERR_ARG, "a reaction names no species");
      d.prodsp[j] = r.prodsp[j], d.prodnu[j] = r.prodnu[j];
    }
    for (int j = 0; j < r.nnet; j++) {
      if (!sp_ok(r.netsp[j])) return fail(PGB_ERR_ARG, "a reaction names no species");
      d.netsp[j] = r.netsp[j], d.netnu[j] = r.netnu[j], d.netnuMW[j] = r.netnuMW[j];
    }
    d.logA = r.logA, d.b = r.b, d.EaR = r.EaR, d.logprA = r.logprA, d.prb = r.prb, d.prEaR = r.prEaR;
    d.nusum = r.nusum;
    (r.product ? product : logform) = true;
  }
  M->logform = logform, M->product = product;
  c->mech = std::move(M);
  c->version++;
  return PGB_OK;
}

int pgb_production(pgb_case *c, long n, const double *rho, const double *Y, const double *T, double *omega) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (!c->mech) return fail(PGB_ERR_STATE, "the case has no mechanism");
  if (n < 0 || (n && (!rho || !Y || !T || !omega))) return fail(PGB_ERR_ARG, "null arrays");
  if (n == 0) return PGB_OK;
  RET(set_current(c));
  const int ns = c->phys.ns;
  const size_t bytes = sizeof(double) * (size_t)n * (2 + 2 * ns);
  double *d = nullptr;
  CK(cudaMallocAsync((void **)&d, bytes, c->stream));
  double *drho = d, *dT = d + n, *dY = d + 2 * n, *dw = d + 2 * n + (size_t)n * ns;
  cudaError_t e = cudaMemcpyAsync(drho, rho, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dY, Y, sizeof(double) * n * ns, cudaMemcpyHostToDevice, c->stream);
  int rc = PGB_OK;
  if (e == cudaSuccess) rc = kPlain[ns - 1].production(n, drho, dY, dT, dw, c->stream);
  if (e == cudaSuccess && rc == PGB_OK)
    e = cudaMemcpyAsync(omega, dw, sizeof(double) * n * ns, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(d, c->stream);
  const cudaError_t s = cudaStreamSynchronize(c->stream);
  if (rc != PGB_OK) return rc;
  if (e != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("production copies: ") + cudaGetErrorString(e));
  if (s != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("production: ") + cudaGetErrorString(s));
  return PGB_OK;
}

int pgb_case_add_block(pgb_case *c, int ni, int nj, int nk, int *blk) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  if (ni < 1 || nj < 1 || nk < 1) return fail(PGB_ERR_ARG, "a block has at least one cell per axis");
  if (ni > 30000 || nj > 30000 || nk > 30000) return fail(PGB_ERR_ARG, "block too large");
  HostBlock B;
  B.nx = ni, B.ny = nj, B.nz = nk;
  c->blocks.push_back(B);
  if (blk) *blk = (int)c->blocks.size() - 1;
  return PGB_OK;
}

int pgb_case_connect(pgb_case *c, int blk, int nface, int nbr, int nbrface) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  if (blk < 0 || blk >= (int)c->blocks.size() || nface < 1 || nface > 6)
    return fail(PGB_ERR_ARG, "no such block face");
  if (nbr >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "no such neighbour");
  if (nbr >= 0) {
    const int a = (nface - 1) / 2;
    if (nbrface != (nface % 2 ? nface + 1 : nface - 1))
      return fail(PGB_ERR_UNSUPPORTED, "only the orientation 123 (low face to high face) is built");
    const HostBlock &B = c->blocks[blk], &N = c->blocks[nbr];
    const int n[3] = {B.nx, B.ny, B.nz}, m[3] = {N.nx, N.ny, N.nz};
    for (int d = 0; d < 3; d++)
      if (d != a && n[d] != m[d]) return fail(PGB_ERR_ARG, "the two faces do not match cell for cell");
  }
  c->blocks[blk].nbr[nface - 1] = nbr;
  if (nbr >= 0) c->blocks[blk].bc[nface - 1] = -1;
  c->blocks[blk].nbrface[nface - 1] = nbrface;
  return PGB_OK;
}

int pgb_case_connect_oriented(pgb_case *c, int blk, int nface, int nbr, const char *orient, const double *rot) {
  if (!c || !orient) return fail(PGB_ERR_ARG, "null argument");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  if (blk < 0 || blk >= (int)c->blocks.size() || nface < 1 || nface > 6)
    return fail(PGB_ERR_ARG, "no such block face");
  if (nbr < 0 || nbr >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "no such neighbour");
  int code[3], seen = 0;
  for (int d = 0; d < 3; d++) {
    if (orient[d] < '1' || orient[d] > '6') return fail(PGB_ERR_ARG, "an orientation is three digits 1-6");
    code[d] = orient[d] - '0';
    seen |= 1 << ((code[d] - 1) % 3);
  }
  if (seen != 7 || orient[3] != '\0') return fail(PGB_ERR_ARG, "the orientation does not name three distinct axes");
  const int a = (nface - 1) / 2;
  HostBlock &B = c->blocks[blk];
  const HostBlock &N = c->blocks[nbr];
  const int n[3] = {B.nx, B.ny, B.nz}, m[3] = {N.nx, N.ny, N.nz};
  for (int d = 0; d < 3; d++)
    if (d != a && n[d] != m[(code[d] - 1) % 3]) return fail(PGB_ERR_ARG, "the two faces do not match cell for cell");
  for (int d = 0; d < 3; d++) B.orient[nface - 1][d] = code[d];
  const int t = (code[a] - 1) % 3;
  const bool flip = code[a] > 3, low = nface % 2 == 1;
  B.nbr[nface - 1] = nbr;
  B.nbrface[nface - 1] = 2 * t + (low == flip ? 1 : 2);
  B.bc[nface - 1] = -1;
  B.rot[nface - 1] = 0;
  if (rot) {
    bool identity = true;
    for (int q = 0; q < 9; q++) identity = identity && std::fabs(rot[q] - (q % 4 == 0 ? 1.0 : 0.0)) <= 1e-14;
    if (!identity) {
      c->rots.insert(c->rots.end(), rot, rot + 9);
      B.rot[nface - 1] = (int)(c->rots.size() / 9);
    }
  }
  return PGB_OK;
}

int pgb_exchange(pgb_case *c, int reg) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (reg < 0 || reg >= c->phys.nregs) return fail(PGB_ERR_ARG, "no such register");
  RET(set_current(c));
  if (c->nhalo) halo_fill_case(c, c->d_reg[c->phys_of[reg]], c->ne, 1);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_case_halo_boxes(pgb_case *c, long long cap, long long *out, long long *nboxes, long long *rest) {
  if (!c || !nboxes || !rest || (cap > 0 && !out)) return fail(PGB_ERR_ARG, "null argument");
  if (c->blocks.empty()) return fail(PGB_ERR_STATE, "no blocks");
  // the blocks' layout is a host computation; finalize repeats it
  if (!c->finalized) layout_blocks(c);
  std::vector<HaloPatch> boxes;
  std::vector<HaloEntry> left;
  build_boxes(c, boxes, left);
  std::map<long long, int> blk_of;
  for (int b = 0; b < (int)c->blocks.size(); b++) blk_of[c->blocks[b].dev.cv] = b;
  *nboxes = (long long)boxes.size();
  *rest = (long long)left.size();
  for (long long q = 0; q < *nboxes && q < cap; q++) {
    const HaloPatch &P = boxes[q];
    const long long v[14] = {blk_of[P.dcv], P.d0,     P.dst[0], P.dst[1], P.dst[2], P.n0, P.n1, P.cells / (P.n0 * P.n1),
                             blk_of[P.scv], P.s0,     P.sst[0], P.sst[1], P.sst[2], P.rot};
    for (int e = 0; e < 14; e++) out[14 * q + e] = v[e];
  }
  return PGB_OK;
}

int pgb_case_halo_entries(pgb_case *c, long long cap, long long *out, long long *n) {
  if (!c || !n || (cap > 0 && !out)) return fail(PGB_ERR_ARG, "null argument");
  if (c->blocks.empty()) return fail(PGB_ERR_STATE, "no blocks");
  // the blocks' layout is a host computation; finalize repeats it
  if (!c->finalized) layout_blocks(c);
  std::vector<HaloEntry> halo;
  std::vector<int2> blk;
  long long l0 = 0;
  build_halo(c, halo, l0, &blk);
  *n = (long long)halo.size();
  for (long long e = 0; e < *n && e < cap; e++) {
    long long *r = out + 6 * e;
    r[0] = blk[e].x, r[1] = halo[e].didx, r[2] = blk[e].y, r[3] = halo[e].sidx, r[4] = halo[e].rot;
    r[5] = e < l0 ? 0 : 1;
  }
  return PGB_OK;
}

int pgb_case_set_exchange(pgb_case *c, long long nsend, const int *send_blk, const int *send_idx, long long nrecv,
                          const int *recv_blk, const int *recv_idx) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->finalized) return fail(PGB_ERR_STATE, "finalize the case before its exchange");
  if (nsend < 0 || nrecv < 0 || (nsend && (!send_blk || !send_idx)) || (nrecv && (!recv_blk || !recv_idx)))
    return fail(PGB_ERR_ARG, "bad exchange lists");
  auto table = [&](long long n, const int *blk, const int *idx, long long *&d_at, int *&d_vol) -> int {
    if (d_at) cudaFree(d_at), d_at = nullptr;
    if (d_vol) cudaFree(d_vol), d_vol = nullptr;
    if (!n) return PGB_OK;
    std::vector<long long> at(n);
    std::vector<int> vol(n);
    for (long long e = 0; e < n; e++) {
      if (blk[e] < 0 || blk[e] >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "exchange cell: no such block");
      const BlockDev &D = c->blocks[blk[e]].dev;
      if (idx[e] < 0 || idx[e] >= D.vol) return fail(PGB_ERR_ARG, "exchange cell: index outside its block");
      at[e] = (long long)c->ne * D.cv + idx[e];
      vol[e] = (int)D.vol;
    }
    CK(cudaMalloc(&d_at, sizeof(long long) * n));
    CK(cudaMalloc(&d_vol, sizeof(int) * n));
    CK(cudaMemcpy(d_at, at.data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_vol, vol.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    return PGB_OK;
  };
  RET(table(nsend, send_blk, send_idx, c->d_xsend, c->d_xsvol));
  RET(table(nrecv, recv_blk, recv_idx, c->d_xrecv, c->d_xrvol));
  c->nxsend = nsend, c->nxrecv = nrecv;
  // a stage reads halo copies once another case fills some of them
  for (auto &g : c->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  return PGB_OK;
}

// the physical register stage s of the current step reads
static int stage_register(pgb_case *c, int s, int path, int &phys) {
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (path < PGB_PATH_BATCHED || path > PGB_PATH_PACKED) return fail(PGB_ERR_ARG, "no such path");
  if (s < 0 || s >= (int)c->stages.size()) return fail(PGB_ERR_ARG, "no such stage");
  if (path == PGB_PATH_BATCHED) phys = c->plans[c->phase][s].qin;
  else phys = c->phys_of[c->stages[s].q];
  return PGB_OK;
}

int pgb_exchange_pack(pgb_case *c, int stage, int path, double *buf) {
  if (!c || (c->nxsend && !buf)) return fail(PGB_ERR_ARG, "null argument");
  int r = 0;
  RET(stage_register(c, stage, path, r));
  if (c->nxsend)
    k_xpack<<<grid_for(c->nxsend, 256), 256, 0, c->stream>>>(c->d_reg[r], c->d_xsend, c->d_xsvol, c->nxsend, c->ne,
                                                             buf);
  CK(cudaGetLastError());
  return PGB_OK;
}

int pgb_exchange_unpack(pgb_case *c, int stage, int path, const double *buf) {
  if (!c || (c->nxrecv && !buf)) return fail(PGB_ERR_ARG, "null argument");
  int r = 0;
  RET(stage_register(c, stage, path, r));
  if (c->nxrecv)
    k_xunpack<<<grid_for(c->nxrecv, 256), 256, 0, c->stream>>>(c->d_reg[r], c->d_xrecv, c->d_xrvol, c->nxrecv, c->ne,
                                                               buf);
  CK(cudaGetLastError());
  return PGB_OK;
}

int pgb_step_stage(pgb_case *c, int s, int path) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (s != c->stage_next) return fail(PGB_ERR_STATE, "stages run in order, from the step's first");
  const bool fused = path == PGB_PATH_BATCHED;
  if (fused && !fused_capable(c)) return fail(PGB_ERR_UNSUPPORTED, "the batched path does not take this case");
  if (path < PGB_PATH_BATCHED || path > PGB_PATH_PACKED) return fail(PGB_ERR_ARG, "no such path");
  if (c->nbcface[0] || sim_df(c->phys.simulator) || c->phys.chemistry == PGB_CHEM_SUBSTEPPED)
    return fail(PGB_ERR_UNSUPPORTED, "a stage at a time takes the cases without boundaries, double flux or substeps");
  // a shard trades Q's halo between stages; the per-block kernels and the
  // fused passes exchange the gradients' first halo layer inside the stage,
  // which a trade of Q does not give them: their viscous shards are refused
  if ((c->nxsend || c->nxrecv) && sim_visc(c->phys.simulator) && !(fused && batched_form(c) == 1))
    return fail(PGB_ERR_UNSUPPORTED, "a viscous shard steps on the batched path's fused stage kernel alone: it "
                                     "forms its gradients from Q's two-deep halo, the others trade them mid-stage");
  RET(prepare(c, fused));
  if (!fused) RET(ensure_scratch(c));
  int count = 0;
  struct Packed {
    pgb_case *c;
    ~Packed() { c->packed = false; }
  } unpack{c};
  c->packed = path == PGB_PATH_PACKED;
  if (fused) {
    const auto &plan = c->plans[c->phase];
    if (s == 0) CK(cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned int) * plan.size(), c->stream));
    RET(c->form == 2 ? launch_react(c, plan[s], count) : launch_fused(c, plan[s], s, count));
    if (s + 1 == (int)plan.size()) {
      c->phase = (c->phase + 1) % c->period;
      c->phys_of = c->maps[c->phase];
    }
  } else {
    const pgb_stage &st = c->stages[s];
    RET(rhs_plain(c, c->phys_of[st.q], c->phys_of[st.dq], count, st.tfrac));
    combine_stage(c, st, count);
  }
  c->stage_next = (s + 1) % (int)c->stages.size();
  CK(cudaGetLastError());
  return PGB_OK;
}

int pgb_case_set_substeps(pgb_case *c, int cap, int bulk, int bins, double eqtol) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  if (c->phys.chemistry != PGB_CHEM_SUBSTEPPED) return fail(PGB_ERR_STATE, "the case's chemistry is not sub-stepped");
  if (cap < 1) return fail(PGB_ERR_ARG, "max-substeps is a count of one or more");
  if (bulk < 1 || bulk > cap) return fail(PGB_ERR_ARG, "bulk-substeps is a count from one to max-substeps");
  if (bins < 1 || bins > 16) return fail(PGB_ERR_ARG, "stiff-bins is a count from one to sixteen");
  if (!(eqtol >= 0.0 && eqtol < 1.0)) return fail(PGB_ERR_ARG, "equilibrium-tolerance is a mass fraction below one");
  SubstepOpts &o = c->subopt;
  o.cap = cap, o.bulk = bulk, o.bins = bins, o.eqtol = eqtol, o.stepfrac = 1e-12;
  // the bulk pass's limit and the bins' spacing in ln(count / limit) (substepped.py:47-52)
  o.limitinv = 1.0 / bulk;
  o.binscale = bulk < cap ? bins / std::log((double)cap / bulk) : 0.0;
  return PGB_OK;
}

int pgb_substeps_get(pgb_case *c, int blk, int *host, long count) {
  if (!c || !host) return fail(PGB_ERR_ARG, "null argument");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "no such block");
  if (!c->d_subs) return fail(PGB_ERR_STATE, "no sub-stepped right-hand side has run");
  const BlockDev &D = c->blocks[blk].dev;
  if (count != (long)D.nx * D.ny * D.nz) return fail(PGB_ERR_ARG, "host array of the wrong size");
  std::vector<int> full((size_t)D.vol);
  CK(cudaMemcpyAsync(full.data(), c->d_subs + D.cv, sizeof(int) * D.vol, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  long q = 0;
  for (int k = 0; k < D.nz; k++)
    for (int j = 0; j < D.ny; j++)
      for (int i = 0; i < D.nx; i++) host[q++] = full[cell_index(D, i + NG, j + NG, k + NG)];
  return PGB_OK;
}

int pgb_stiff_head(pgb_case *c, unsigned int *head, int n) {
  if (!c || !head) return fail(PGB_ERR_ARG, "null argument");
  if (!c->d_stiffhead) return fail(PGB_ERR_STATE, "no sub-stepped right-hand side has run");
  if (n < 1 || n > c->subopt.bins + 1) return fail(PGB_ERR_ARG, "the header holds bins + 1 counts");
  CK(cudaMemcpyAsync(head, c->d_stiffhead, sizeof(unsigned int) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_case_add_bc(pgb_case *c, int kind, const int *ops, const double *args, const int *starts, int nvalues,
                    int *id) {
  if (!c || !id || !starts || (nvalues && (!ops || !args))) return fail(PGB_ERR_ARG, "null argument");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  if (kind < 1 || kind >= PGB_BC_NKINDS) return fail(PGB_ERR_ARG, "no such boundary kind");
  const bool ns_only = kind >= PGB_BC_NOSLIP_ADIA_WALL && kind <= PGB_BC_MOV_ISOT_WALL;
  if (ns_only && !sim_visc(c->phys.simulator))
    return fail(PGB_ERR_ARG, "the no-slip and moving walls are the navier-stokes simulator's kinds");
  const int want = bc_head_values(kind) + (bc_is_inlet(kind) ? c->phys.ns - 1 : 0);
  if (nvalues != want) return fail(PGB_ERR_ARG, "the entry gives another number of values than its kind reads");
  if (starts[0] < 0) return fail(PGB_ERR_ARG, "a negative program start");
  const int total = starts[nvalues] - starts[0];
  if (total < 0 || (long long)c->bc_ops.size() + total > PGB_BC_MAXOPS)
    return fail(PGB_ERR_ARG, "the boundary programs are longer than the build takes");
  BcEntry E{};
  E.kind = kind;
  E.nval = nvalues;
  const int base = (int)c->bc_ops.size();
  for (int v = 0; v < nvalues; v++) {
    if (starts[v + 1] < starts[v]) return fail(PGB_ERR_ARG, "program starts out of order");
    // each program is checked on a model of the device's stack
    int depth = 0;
    for (int k = starts[v]; k < starts[v + 1]; k++) {
      const int op = ops[k];
      if (op < 0 || op >= PGB_NOPS) return fail(PGB_ERR_ARG, "no such program operation");
      if (op <= PGB_OP_T) {
        if (++depth > PGB_BC_STACK) return fail(PGB_ERR_ARG, "a boundary program deeper than its stack");
        continue;
      }
      const bool binary = op == PGB_OP_ADD || op == PGB_OP_SUB || op == PGB_OP_MUL || op == PGB_OP_DIV ||
                          op == PGB_OP_POW || op == PGB_OP_MIN || op == PGB_OP_MAX;
      if (depth < (binary ? 2 : 1)) return fail(PGB_ERR_ARG, "a boundary program takes more than it has");
      if (binary) depth--;
    }
    if (depth != 1) return fail(PGB_ERR_ARG, "a boundary program must leave one value");
  }
  for (int v = 0; v <= nvalues; v++) E.start[v] = base + starts[v] - starts[0];
  for (int k = starts[0]; k < starts[nvalues]; k++) c->bc_ops.push_back(BcOp{ops[k], 0, args[k]});
  *id = (int)c->bc_entries.size();
  c->bc_entries.push_back(E);
  return PGB_OK;
}

int pgb_case_set_face_bc(pgb_case *c, int blk, int nface, int bc) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  if (blk < 0 || blk >= (int)c->blocks.size() || nface < 1 || nface > 6)
    return fail(PGB_ERR_ARG, "no such block face");
  if (bc < 0 || bc >= (int)c->bc_entries.size()) return fail(PGB_ERR_ARG, "no such boundary entry");
  if (c->blocks[blk].nbr[nface - 1] >= 0) return fail(PGB_ERR_ARG, "the face joins a neighbour; it is no boundary");
  c->blocks[blk].bc[nface - 1] = bc;
  return PGB_OK;
}

int pgb_set_time(pgb_case *c, double t) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  k_setscalar<<<1, 1, 0, c->stream>>>(c->d_clock, t);
  CK(cudaGetLastError());
  return PGB_OK;
}

int pgb_get_time(pgb_case *c, double *t) {
  if (!c || !t) return fail(PGB_ERR_ARG, "null argument");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  CK(cudaMemcpyAsync(t, c->d_clock, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_case_set_stages(pgb_case *c, const pgb_stage *stages, int nstages) {
  if (!c || !stages || nstages < 1 || nstages > 8) return fail(PGB_ERR_ARG, "bad stages");
  for (int s = 0; s < nstages; s++) {
    const pgb_stage &st = stages[s];
    auto okreg = [&](int r) { return r >= -1 && r < c->phys.nregs; };
    if (!okreg(st.q) || st.q < 0 || !okreg(st.dq) || st.dq < 0 || st.ncombine < 1 || st.ncombine > 2)
      return fail(PGB_ERR_ARG, "bad stage");
    for (int m = 0; m < st.ncombine; m++) {
      const pgb_combine &cb = st.combine[m];
      if (cb.out < 0 || cb.out >= c->phys.nregs || cb.nterms < 1 || cb.nterms > 3) return fail(PGB_ERR_ARG, "bad combine");
      for (int n = 0; n < cb.nterms; n++)
        if (!okreg(cb.reg[n])) return fail(PGB_ERR_ARG, "bad combine register");
    }
  }
  if (c->finalized) return fail(PGB_ERR_STATE, "stages are set before finalize");
  c->stages.assign(stages, stages + nstages);
  return PGB_OK;
}

int pgb_case_set_halo_pull(pgb_case *c, int on) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  c->pull_want = on != 0;
  for (auto &g : c->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  return PGB_OK;
}

int pgb_case_halo_pull(const pgb_case *c, int *on) {
  if (!c || !on) return fail(PGB_ERR_ARG, "null argument");
  // before finalize a host computation: whether the wish and the faces allow it
  *on = c->finalized ? (pulls(c) ? 1 : 0) : (c->pull_want && faces_pullable(c) ? 1 : 0);
  return PGB_OK;
}

int pgb_case_set_generated_chemistry(pgb_case *c, int on) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (c->finalized) return fail(PGB_ERR_STATE, "the case is finalized");
  c->gen_want = on != 0;
  return PGB_OK;
}

int pgb_case_generated_chemistry(const pgb_case *c, int *on, char *why, long long cap) {
  if (!c || !on) return fail(PGB_ERR_ARG, "null argument");
  *on = c->gen_src != nullptr;
  if (why && cap > 0) {
    const size_t n = std::min<size_t>((size_t)cap - 1, c->gen_why.size());
    std::memcpy(why, c->gen_why.data(), n);
    why[n] = 0;
  }
  return PGB_OK;
}

int pgb_case_rates_source(pgb_case *c, char *buf, long long cap, long long *len) {
  if (!c || !len || (cap > 0 && !buf)) return fail(PGB_ERR_ARG, "null argument");
  if (!c->mech) return fail(PGB_ERR_STATE, "the case has no mechanism");
  if (!c->finalized) RET(build_species(c));
  const std::string src = rates_source(*c->mech, c->sp, c->phys.ns);
  *len = (long long)src.size();
  if (buf && cap > 0) {
    const size_t n = std::min<size_t>((size_t)cap - 1, src.size());
    std::memcpy(buf, src.data(), n);
    buf[n] = 0;
  }
  return PGB_OK;
}

int pgb_case_rates_compile(pgb_case *c, char *log, long long cap) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->mech) return fail(PGB_ERR_STATE, "the case has no mechanism");
  if (!c->finalized) RET(build_species(c));
  std::string cubin, err;
  const bool ok = rates_compile(rates_source(*c->mech, c->sp, c->phys.ns), cubin, err);
  if (log && cap > 0) {
    const size_t n = std::min<size_t>((size_t)cap - 1, err.size());
    std::memcpy(log, err.data(), n);
    log[n] = 0;
  }
  return ok ? PGB_OK : fail(PGB_ERR_UNSUPPORTED, err);
}

int pgb_case_finalize(pgb_case *c) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (c->finalized) return PGB_OK;
  if (c->blocks.empty()) return fail(PGB_ERR_STATE, "no blocks");
  if (c->stages.empty()) return fail(PGB_ERR_STATE, "no stages");
  RET(build_species(c));
  if (!c->stream) CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  RET(build_generated(c));
  if (!c->ev0) CK(cudaEventCreate(&c->ev0));
  if (!c->ev1) CK(cudaEventCreate(&c->ev1));
  c->cells = layout_blocks(c);
  c->pull_faces = faces_pullable(c);
  if (c->pull_faces) {
    // the block reached from b by a step of (di, dj, dk), i first, then j,
    // then k, as a halo cell's source is located
    std::vector<int> t(27 * c->blocks.size());
    for (int b = 0; b < (int)c->blocks.size(); b++)
      for (int dk = -1; dk <= 1; dk++)
        for (int dj = -1; dj <= 1; dj++)
          for (int di = -1; di <= 1; di++) {
            int s = b;
            if (di) s = c->blocks[s].nbr[di < 0 ? 0 : 1];
            if (dj) s = c->blocks[s].nbr[dj < 0 ? 2 : 3];
            if (dk) s = c->blocks[s].nbr[dk < 0 ? 4 : 5];
            t[27 * b + 9 * (dk + 1) + 3 * (dj + 1) + di + 1] = s;
          }
    CK(cudaMalloc(&c->d_nbr27, sizeof(int) * t.size()));
    CK(cudaMemcpy(c->d_nbr27, t.data(), sizeof(int) * t.size(), cudaMemcpyHostToDevice));
  }
  c->interior_cells = 0;
  for (auto &B : c->blocks) c->interior_cells += (long long)B.nx * B.ny * B.nz;
  const size_t n = (size_t)c->cells;
  for (int r = 0; r < c->phys.nregs; r++) {
    CK(cudaMalloc(&c->d_reg[r], sizeof(double) * c->ne * n));
    CK(cudaMemsetAsync(c->d_reg[r], 0, sizeof(double) * c->ne * n, c->stream));
  }
  CK(cudaMalloc(&c->d_met, sizeof(double) * M_NCOMP * n));
  CK(cudaMemsetAsync(c->d_met, 0, sizeof(double) * M_NCOMP * n, c->stream));
  CK(cudaMalloc(&c->d_dt, sizeof(double)));
  // the step scalar is nothing until a step sets it (a right-hand side
  // before any step integrates the chemistry over no time)
  CK(cudaMemsetAsync(c->d_dt, 0, sizeof(double), c->stream));
  CK(cudaMalloc(&c->d_clock, sizeof(double)));
  CK(cudaMemsetAsync(c->d_clock, 0, sizeof(double), c->stream));
  CK(cudaMalloc(&c->d_one, sizeof(double)));
  k_setscalar<<<1, 1, 0, c->stream>>>(c->d_one, 1.0);
  CK(cudaGetLastError());
  CK(cudaMalloc(&c->d_cfl, sizeof(double) * 3));
  CK(cudaMemsetAsync(c->d_cfl, 0, sizeof(double) * 3, c->stream));
  CK(cudaMalloc(&c->d_ctrl, sizeof(double) * 2));
  RET(build_bcs(c));
  CK(cudaMalloc(&c->d_counter, sizeof(unsigned int) * 16));
  CK(cudaMalloc(&c->d_blks, sizeof(BlockDev) * c->blocks.size()));
  std::vector<BlockDev> devs;
  for (auto &B : c->blocks) devs.push_back(B.dev);
  CK(cudaMemcpy(c->d_blks, devs.data(), sizeof(BlockDev) * devs.size(), cudaMemcpyHostToDevice));
  std::vector<HaloEntry> halo;
  build_halo(c, halo, c->nhalo_l0);
  c->nhalo = (long long)halo.size();
  CK(cudaMalloc(&c->d_halo, sizeof(HaloEntry) * std::max<size_t>(1, halo.size())));
  CK(cudaMemcpy(c->d_halo, halo.data(), sizeof(HaloEntry) * halo.size(), cudaMemcpyHostToDevice));
  {
    // the boxes, used only when they hold exactly the listed cells
    std::vector<HaloPatch> boxes;
    std::vector<HaloEntry> rest;
    build_boxes(c, boxes, rest);
    long long cells = (long long)rest.size();
    for (const HaloPatch &P : boxes) cells += P.cells;
    if (!boxes.empty() && cells == c->nhalo) {
      std::vector<int2> cta;
      for (int q = 0; q < (int)boxes.size(); q++)
        for (int t = 0; t < (boxes[q].cells + 255) / 256; t++) cta.push_back(make_int2(q, t));
      for (int t = 0; t < (int)((rest.size() + 255) / 256); t++) cta.push_back(make_int2(-1, t));
      CK(cudaMalloc(&c->d_boxes, sizeof(HaloPatch) * boxes.size()));
      CK(cudaMemcpy(c->d_boxes, boxes.data(), sizeof(HaloPatch) * boxes.size(), cudaMemcpyHostToDevice));
      CK(cudaMalloc(&c->d_boxcta, sizeof(int2) * cta.size()));
      CK(cudaMemcpy(c->d_boxcta, cta.data(), sizeof(int2) * cta.size(), cudaMemcpyHostToDevice));
      if (!rest.empty()) {
        CK(cudaMalloc(&c->d_boxrest, sizeof(HaloEntry) * rest.size()));
        CK(cudaMemcpy(c->d_boxrest, rest.data(), sizeof(HaloEntry) * rest.size(), cudaMemcpyHostToDevice));
      }
      c->nboxcta = (long long)cta.size();
      c->nboxrest = (long long)rest.size();
    }
  }
  if (!c->rots.empty()) {
    CK(cudaMalloc(&c->d_rots, sizeof(double) * c->rots.size()));
    CK(cudaMemcpy(c->d_rots, c->rots.data(), sizeof(double) * c->rots.size(), cudaMemcpyHostToDevice));
  }
  CK(cudaStreamSynchronize(c->stream));
  c->finalized = true;
  RET(build_plans(c));
  return PGB_OK;
}

int pgb_case_halo(const pgb_case *c, int *ng) {
  if (!c || !ng) return fail(PGB_ERR_ARG, "null argument");
  *ng = NG;
  return PGB_OK;
}

int pgb_case_device_bytes(const pgb_case *c, size_t *bytes) {
  if (!c || !bytes) return fail(PGB_ERR_ARG, "null argument");
  const size_t n = (size_t)c->cells;
  size_t b = sizeof(double) * n * ((size_t)c->ne * c->phys.nregs + M_NCOMP);
  if (c->d_state) b += sizeof(double) * n * (8 + 2 + 2 * c->phys.ns + 3 * (c->ne - 1) + 3 * c->ne);
  *bytes = b + sizeof(HaloEntry) * (size_t)c->nhalo;
  return PGB_OK;
}

int pgb_metric_set(pgb_case *c, int blk, int which, const double *host, long count) {
  if (!c || !host) return fail(PGB_ERR_ARG, "null argument");
  if (!c->finalized) return fail(PGB_ERR_STATE, "finalize the case before setting metrics");
  if (blk < 0 || blk >= (int)c->blocks.size() || which < 0 || which >= PGB_NMETRICS)
    return fail(PGB_ERR_ARG, "no such block or metric");
  HostBlock &B = c->blocks[blk];
  const BlockDev &D = B.dev;
  static const int comps[PGB_NMETRICS] = {3, 1, 9, 3, 3, 3, 3, 3, 3};
  static const int first[PGB_NMETRICS] = {M_XCC, M_DETJINV, M_JINV, M_S, M_S + 3, M_S + 6, M_XF, M_XF + 3, M_XF + 6};
  const int face = which >= PGB_ARR_IS ? (which - PGB_ARR_IS) % 3 : -1;
  const int X = D.X + (face == 0), Y = D.Y + (face == 1), Z = D.Z + (face == 2);
  const int nc = comps[which];
  if (count != (long)X * Y * Z * nc) return fail(PGB_ERR_ARG, "metric array of the wrong size");
  // host F order [comp][k][j][i] over the array's own extents; the face
  // array's last plane (past the last halo cell) is never read and is dropped
  std::vector<double> dev((size_t)nc * D.vol);
  for (int q = 0; q < nc; q++)
    for (int k = 0; k < D.Z; k++)
      for (int j = 0; j < D.Y; j++)
        for (int i = 0; i < D.X; i++)
          dev[(size_t)q * D.vol + cell_index(D, i, j, k)] = host[(((size_t)q * Z + k) * Y + j) * X + i];
  CK(cudaMemcpy(c->d_met + (size_t)M_NCOMP * D.cv + (size_t)first[which] * D.vol, dev.data(),
                sizeof(double) * dev.size(), cudaMemcpyHostToDevice));
  B.metrics_set[which] = true;
  c->uniform_done = false;
  for (auto &g : c->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  return PGB_OK;
}

static int check_reg(pgb_case *c, int blk, int reg, long count, int comps) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "no such block");
  if (reg < 0 || reg >= c->phys.nregs) return fail(PGB_ERR_ARG, "no such register");
  const BlockDev &D = c->blocks[blk].dev;
  if (count != (long)D.nx * D.ny * D.nz * comps) return fail(PGB_ERR_ARG, "host array of the wrong size");
  return PGB_OK;
}

static int stage_host(pgb_case *c, long long n) {
  if (n > c->prims_cap) {
    if (c->d_prims) cudaFree(c->d_prims);
    c->d_prims = nullptr;
    CK(cudaMalloc(&c->d_prims, sizeof(double) * n));
    c->prims_cap = n;
  }
  return PGB_OK;
}

int pgb_array_set(pgb_case *c, int blk, int reg, const double *host, long count) {
  RET(check_reg(c, blk, reg, count, c->ne));
  if (!host) return fail(PGB_ERR_ARG, "null host array");
  RET(stage_host(c, count));
  CK(cudaMemcpyAsync(c->d_prims, host, sizeof(double) * count, cudaMemcpyHostToDevice, c->stream));
  const BlockDev &D = c->blocks[blk].dev;
  k_unpack<<<grid_for((long long)D.nx * D.ny * D.nz, 256), 256, 0, c->stream>>>(c->d_blks, blk, c->ne, c->d_prims,
                                                                                   c->d_reg[c->phys_of[reg]]);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_array_get(pgb_case *c, int blk, int reg, double *host, long count) {
  RET(check_reg(c, blk, reg, count, c->ne));
  if (!host) return fail(PGB_ERR_ARG, "null host array");
  RET(stage_host(c, count));
  const BlockDev &D = c->blocks[blk].dev;
  k_pack<<<grid_for((long long)D.nx * D.ny * D.nz, 256), 256, 0, c->stream>>>(c->d_blks, blk, c->ne,
                                                                                 c->d_reg[c->phys_of[reg]], c->d_prims);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, c->d_prims, sizeof(double) * count, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_array_get_full(pgb_case *c, int blk, int reg, double *host, long count) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "no such block");
  if (reg < 0 || reg >= c->phys.nregs) return fail(PGB_ERR_ARG, "no such register");
  if (!host) return fail(PGB_ERR_ARG, "null host array");
  const BlockDev &D = c->blocks[blk].dev;
  if (count != (long)D.vol * c->ne) return fail(PGB_ERR_ARG, "host array of the wrong size");
  // a block's register is its components' full arrays end to end: F order already
  CK(cudaMemcpyAsync(host, c->d_reg[c->phys_of[reg]] + (size_t)c->ne * D.cv, sizeof(double) * count,
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

// one field of a block's eos state over its full extents, F order: the
// state the last right-hand side (or set_prims) formed, each cell's
// (p, T, rhoinv, rho, e, cp, gamma, c), the real gas's Z, the double flux's
// plane (theta, eps, kappa, zeta...) (the reference's state array,
// peregrine/simulator/euler/simulator.py:66-90 reads p and T from it)
int pgb_eos_get(pgb_case *c, int blk, int field, double *host, long count) {
  if (!c || !host) return fail(PGB_ERR_ARG, "null argument");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (blk < 0 || blk >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "no such block");
  if (field < 0 || field >= SW) return fail(PGB_ERR_ARG, "no such state field");
  const BlockDev &D = c->blocks[blk].dev;
  if (count != (long)D.vol) return fail(PGB_ERR_ARG, "host array of the wrong size");
  if (!c->d_state) return fail(PGB_ERR_STATE, "no state yet: set the primitives first");
  if (c->state_stale) return fail(PGB_ERR_STATE, "the batched path forms the state in registers and keeps none");
  RET(set_current(c));
  CK(cudaMemcpyAsync(host, c->d_state + (size_t)SW * D.cv + (size_t)field * D.vol, sizeof(double) * count,
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_set_prims(pgb_case *c, int blk, int reg, const double *host, long count) {
  RET(check_reg(c, blk, reg, count, c->ne));
  if (!host) return fail(PGB_ERR_ARG, "null host array");
  RET(set_current(c));
  RET(ensure_state(c));
  RET(stage_host(c, count));
  CK(cudaMemcpyAsync(c->d_prims, host, sizeof(double) * count, cudaMemcpyHostToDevice, c->stream));
  std::vector<BlockDev> hb;
  const PlainCase pc = plain_case(c, hb);
  RET(kPlain[c->phys.ns - 1].fromprims(&pc, blk, c->d_prims, c->d_reg[c->phys_of[reg]]));
  c->state_stale = false;
  // a halo cell's first Newton starts from the stored T of the cell it copies
  if (c->nhalo) halo_fill_case(c, c->d_state, SW, HALO_SCALARS);
  c->df_fresh = true;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_advance(pgb_case *c, int n) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  RET(prepare(c, false));
  if (n < 0 || n >= (int)c->stages.size()) return fail(PGB_ERR_ARG, "no such stage");
  int count = 0;
  combine_stage(c, c->stages[n], count);
  CK(cudaGetLastError());
  return PGB_OK;
}

int pgb_rhs(pgb_case *c, int q, int dq) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  RET(prepare(c, false));
  if (q < 0 || q >= c->phys.nregs || dq < 0 || dq >= c->phys.nregs || q == dq)
    return fail(PGB_ERR_ARG, "bad registers");
  int count = 0;
  // the double flux's planes, frozen once after the state was set
  RET(df_settle(c, c->phys_of[q]));
  RET(rhs_plain(c, c->phys_of[q], c->phys_of[dq], count));
  return PGB_OK;
}

int pgb_rhs_path(pgb_case *c, int q, int dq, int path) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (path < PGB_PATH_BATCHED || path > PGB_PATH_PACKED) return fail(PGB_ERR_ARG, "no such path");
  if (path != PGB_PATH_BATCHED) {
    struct Packed {
      pgb_case *c;
      ~Packed() { c->packed = false; }
    } unpack{c};
    c->packed = path == PGB_PATH_PACKED;
    return pgb_rhs(c, q, dq);
  }
  if (!fused_capable(c)) return fail(PGB_ERR_UNSUPPORTED, "the batched path does not take this case");
  if (q < 0 || q >= c->phys.nregs || dq < 0 || dq >= c->phys.nregs || q == dq)
    return fail(PGB_ERR_ARG, "bad registers");
  RET(prepare(c, true));
  if (c->form == 2) RET(df_settle(c, c->phys_of[q]));
  int count = 0;
  RET(rhs_fused(c, c->phys_of[q], c->phys_of[dq], count));
  CK(cudaGetLastError());
  return PGB_OK;
}

// nsteps steps at the step size in d_dt (or the cfl controller's, with
// ctrl_cfl): whole graph units while they fit, single steps after
static int step_loop(pgb_case *c, int nsteps, int path, int graph) {
  const bool fused = path == PGB_PATH_BATCHED;
  // the per-block kernels packed: each pass one launch over every block
  struct Packed {
    pgb_case *c;
    ~Packed() { c->packed = false; }
  } unpack{c};
  c->packed = path == PGB_PATH_PACKED;
  CK(cudaEventRecord(c->ev0, c->stream));
  int done = 0;
  while (done < nsteps) {
    const int unit = fused ? c->period : 1;
    if (graph && c->phase == 0 && nsteps - done >= unit) {
      cudaGraphExec_t &ge = c->graph[path];
      if (ge && (c->graph_map[path] != c->phys_of || c->graph_cfl[path] != c->ctrl_cfl)) {
        cudaGraphExecDestroy(ge);
        ge = nullptr;
      }
      if (!ge) {
        c->graph_map[path] = c->phys_of;
        c->graph_cfl[path] = c->ctrl_cfl;
        cudaGraph_t g;
        int count = 0;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        int rc = PGB_OK;
        for (int u = 0; u < unit && rc == PGB_OK; u++) rc = fused ? step_fused(c, count) : step_plain(c, count);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (rc != PGB_OK) return rc;
        if (e != cudaSuccess) return fail(PGB_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        CK(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
        c->launches[path] = count / unit;
        // the capture advanced the phase as the launches will
        c->phase = 0;
        c->phys_of = c->maps.empty() ? c->phys_of : c->maps[0];
      }
      CK(cudaGraphLaunch(ge, c->stream));
      if (fused) {
        c->phase = 0;
        c->phys_of = c->maps[0];
      }
      done += unit;
      continue;
    }
    int count = 0;
    RET(fused ? step_fused(c, count) : step_plain(c, count));
    c->launches[path] = count;
    done += 1;
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  return PGB_OK;
}

static int step_begin(pgb_case *c, int nsteps, int path) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (c->stage_next != 0) return fail(PGB_ERR_STATE, "a step taken stage by stage is not finished");
  if (nsteps < 0) return fail(PGB_ERR_ARG, "negative step count");
  if (path < PGB_PATH_BATCHED || path > PGB_PATH_PACKED) return fail(PGB_ERR_ARG, "no such path");
  const bool fused = path == PGB_PATH_BATCHED;
  if (fused && !fused_capable(c))
    return fail(PGB_ERR_UNSUPPORTED, "the batched path takes the single-species cpg kepaec case; use the per-block path");
  RET(prepare(c, fused));
  if (!fused) RET(ensure_scratch(c));
  if ((!fused || c->form == 2) && !c->stages.empty()) RET(df_settle(c, c->phys_of[c->stages[0].q]));
  return PGB_OK;
}

int pgb_step(pgb_case *c, double dt, int nsteps, int path, int graph) {
  RET(step_begin(c, nsteps, path));
  k_setscalar<<<1, 1, 0, c->stream>>>(c->d_dt, dt);
  CK(cudaGetLastError());
  c->ctrl_cfl = false;
  return step_loop(c, nsteps, path, graph);
}

int pgb_step_cfl(pgb_case *c, double cfl, double dtmax, int nsteps, int path, int graph) {
  if (!(cfl > 0.0) || !(dtmax > 0.0)) return fail(PGB_ERR_ARG, "cfl and dt-max are positive");
  RET(step_begin(c, nsteps, path));
  k_setscalar<<<1, 1, 0, c->stream>>>(c->d_ctrl, cfl);
  k_setscalar<<<1, 1, 0, c->stream>>>(c->d_ctrl + 1, dtmax);
  CK(cudaGetLastError());
  c->ctrl_cfl = true;
  const int rc = step_loop(c, nsteps, path, graph);
  c->ctrl_cfl = false;
  return rc;
}

int pgb_cflmax(pgb_case *c, int reg, double *out) {
  if (!c || !out) return fail(PGB_ERR_ARG, "null argument");
  RET(prepare(c, false));
  if (reg < 0 || reg >= c->phys.nregs) return fail(PGB_ERR_ARG, "no such register");
  int count = 0;
  RET(cfl_pass(c, c->phys_of[reg], count));
  CK(cudaMemcpyAsync(out, c->d_cfl, sizeof(double) * 3, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_set_dt(pgb_case *c, double dt) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  k_setscalar<<<1, 1, 0, c->stream>>>(c->d_dt, dt);
  CK(cudaGetLastError());
  return PGB_OK;
}

int pgb_last_dt(pgb_case *c, double *dt) {
  if (!c || !dt) return fail(PGB_ERR_ARG, "null argument");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  CK(cudaMemcpyAsync(dt, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_step_timed(pgb_case *c, double dt, int nsteps, int path, float *ms, int *kind, int cap, int *n) {
  if (!c || !n || (cap > 0 && (!ms || !kind))) return fail(PGB_ERR_ARG, "null argument");
  if (path < PGB_PATH_BATCHED || path > PGB_PATH_PACKED) return fail(PGB_ERR_ARG, "no such path");
  const bool fused = path == PGB_PATH_BATCHED;
  if (fused && !fused_capable(c)) return fail(PGB_ERR_UNSUPPORTED, "the batched path does not take this case");
  RET(prepare(c, fused));
  if (!fused) RET(ensure_scratch(c));
  if ((!fused || c->form == 2) && !c->stages.empty()) RET(df_settle(c, c->phys_of[c->stages[0].q]));
  k_setscalar<<<1, 1, 0, c->stream>>>(c->d_dt, dt);
  CK(cudaGetLastError());
  c->timing = true;
  c->tnext = 0;
  c->tkind.clear();
  c->packed = path == PGB_PATH_PACKED;
  CK(cudaEventRecord(c->ev0, c->stream));
  int rc = PGB_OK;
  for (int s = 0; s < nsteps && rc == PGB_OK; s++) {
    int count = 0;
    rc = fused ? step_fused(c, count) : step_plain(c, count);
    c->launches[path] = count;
  }
  c->timing = false;
  c->packed = false;
  if (rc != PGB_OK) return rc;
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  const int total = (int)c->tnext;
  *n = total;
  for (int q = 0; q < total && q < cap; q++) {
    // a launch's time: from the event before it (the previous launch's, or
    // the start) to its own; the memset nodes between steps fall in the first
    // launch of each step
    cudaEvent_t before = q == 0 ? c->ev0 : c->tev[q - 1];
    CK(cudaEventElapsedTime(&ms[q], before, c->tev[q]));
    kind[q] = c->tkind[q];
  }
  return PGB_OK;
}

int pgb_state_set(pgb_case *c, int reg, const double *host, long count) {
  if (!c || !host) return fail(PGB_ERR_ARG, "null argument");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (reg < 0 || reg >= c->phys.nregs) return fail(PGB_ERR_ARG, "no such register");
  long long inner = 0;
  for (auto &B : c->blocks) inner += (long long)B.nx * B.ny * B.nz;
  if (count != inner * c->ne) return fail(PGB_ERR_ARG, "host state of the wrong size");
  if (count > c->stage_cap) {
    if (c->d_stage) cudaFree(c->d_stage);
    c->d_stage = nullptr;
    CK(cudaMalloc(&c->d_stage, sizeof(double) * count));
    c->stage_cap = count;
  }
  CK(cudaMemcpyAsync(c->d_stage, host, sizeof(double) * count, cudaMemcpyHostToDevice, c->stream));
  long long at = 0;
  for (int b = 0; b < (int)c->blocks.size(); b++) {
    const BlockDev &D = c->blocks[b].dev;
    const long long n = (long long)D.nx * D.ny * D.nz;
    k_unpack<<<grid_for(n, 256), 256, 0, c->stream>>>(c->d_blks, b, c->ne, c->d_stage + at, c->d_reg[c->phys_of[reg]]);
    at += n * c->ne;
  }
  CK(cudaGetLastError());
  return PGB_OK;
}

int pgb_state_get(pgb_case *c, int reg, double *host, long count) {
  if (!c || !host) return fail(PGB_ERR_ARG, "null argument");
  if (!c->finalized) return fail(PGB_ERR_STATE, "the case is not finalized");
  if (reg < 0 || reg >= c->phys.nregs) return fail(PGB_ERR_ARG, "no such register");
  long long inner = 0;
  for (auto &B : c->blocks) inner += (long long)B.nx * B.ny * B.nz;
  if (count != inner * c->ne) return fail(PGB_ERR_ARG, "host state of the wrong size");
  if (count > c->stage_cap) {
    if (c->d_stage) cudaFree(c->d_stage);
    c->d_stage = nullptr;
    CK(cudaMalloc(&c->d_stage, sizeof(double) * count));
    c->stage_cap = count;
  }
  long long at = 0;
  for (int b = 0; b < (int)c->blocks.size(); b++) {
    const BlockDev &D = c->blocks[b].dev;
    const long long n = (long long)D.nx * D.ny * D.nz;
    k_pack<<<grid_for(n, 256), 256, 0, c->stream>>>(c->d_blks, b, c->ne, c->d_reg[c->phys_of[reg]], c->d_stage + at);
    at += n * c->ne;
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, c->d_stage, sizeof(double) * count, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGB_OK;
}

int pgb_host_register(void *host, size_t bytes) {
  if (!host || !bytes) return fail(PGB_ERR_ARG, "null argument");
  CK(cudaHostRegister(host, bytes, cudaHostRegisterDefault));
  return PGB_OK;
}

int pgb_host_unregister(void *host) {
  if (!host) return fail(PGB_ERR_ARG, "null argument");
  CK(cudaHostUnregister(host));
  return PGB_OK;
}

int pgb_case_stream(const pgb_case *c, void **stream) {
  if (!c || !stream) return fail(PGB_ERR_ARG, "null argument");
  *stream = (void *)c->stream;
  return PGB_OK;
}

int pgb_last_step_ms(const pgb_case *c, float *ms) {
  if (!c || !ms) return fail(PGB_ERR_ARG, "null argument");
  CK(cudaEventSynchronize(c->ev1));
  CK(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return PGB_OK;
}

int pgb_launches_per_step(const pgb_case *c, int path, int *count) {
  if (!c || !count || path < 0 || path > PGB_PATH_PACKED) return fail(PGB_ERR_ARG, "bad argument");
  *count = c->launches[path];
  return PGB_OK;
}

int pgb_set_tile(pgb_case *c, int blk, int tw, int th, int kchunk) {
  if (!c || blk < 0 || blk >= (int)c->blocks.size()) return fail(PGB_ERR_ARG, "no such block");
  // a tile the fused kernel of the case cannot take is replaced by its
  // default when the work list is built
  HostBlock &B = c->blocks[blk];
  if (tw == 0 && th == 0) {
    // back to the default tile of the case's kernel
    B.tw = 0;
    c->tiles_dirty = true;
    for (auto &g : c->graph)
      if (g) cudaGraphExecDestroy(g), g = nullptr;
    return PGB_OK;
  }
  if (tw < 1 || th < 1 || kchunk < 1) return fail(PGB_ERR_ARG, "bad tile");
  B.tw = std::min(tw, B.nx), B.th = std::min(th, B.ny), B.kchunk = std::min(kchunk, B.nz);
  c->tiles_dirty = true;
  for (auto &g : c->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  return PGB_OK;
}

int pgb_get_tile(const pgb_case *c, int blk, int *tw, int *th, int *kchunk) {
  if (!c || blk < 0 || blk >= (int)c->blocks.size() || !tw || !th || !kchunk) return fail(PGB_ERR_ARG, "bad argument");
  HostBlock B = c->blocks[blk];
  if (B.tw <= 0) {
    if (c->use_v2) default_tile2(B, kV2[c->v2]);
    else default_tile(B);
  }
  *tw = B.tw, *th = B.th, *kchunk = B.kchunk;
  return PGB_OK;
}

int pgb_set_fused_shape(pgb_case *c, int threads, int minblocks, int width) {
  if (!c) return fail(PGB_ERR_ARG, "null case");
  int pick = -1;
  for (int q = 0; q < kNV2; q++)
    if (kV2[q].nt == threads && kV2[q].minb == minblocks && kV2[q].tw == width) pick = q;
  if (pick < 0) {
    std::string have;
    for (int q = 0; q < kNV2; q++)
      have += " " + std::to_string(kV2[q].nt) + "x" + std::to_string(kV2[q].minb) + "x" + std::to_string(kV2[q].tw);
    return fail(PGB_ERR_ARG, "no uniform kernel of that shape; threads x minblocks x width:" + have);
  }
  if (pick != c->v2)
    for (auto &B : c->blocks) B.tw = 0;
  c->v2 = pick;
  c->tiles_dirty = true;
  for (auto &g : c->graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
  return PGB_OK;
}

int pgb_fused_shapes(int *shapes, int cap, int *n) {
  if (!n || (cap > 0 && !shapes)) return fail(PGB_ERR_ARG, "null argument");
  *n = kNV2;
  for (int q = 0; q < kNV2 && q < cap; q++) {
    shapes[4 * q] = kV2[q].nt, shapes[4 * q + 1] = kV2[q].minb;
    shapes[4 * q + 2] = kV2[q].tw, shapes[4 * q + 3] = kV2[q].th;
  }
  return PGB_OK;
}

int pgb_case_batched_form(const pgb_case *c, int *form) {
  if (!c || !form) return fail(PGB_ERR_ARG, "null argument");
  *form = batched_form(c);
  return PGB_OK;
}

int pgb_block_uniform(const pgb_case *c, int blk, int *uniform) {
  if (!c || blk < 0 || blk >= (int)c->blocks.size() || !uniform) return fail(PGB_ERR_ARG, "bad argument");
  *uniform = c->blocks[blk].dev.uniform;
  return PGB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The serving pool: independent cases, each one periodic block, admitted into
// one device arena while others run, advanced together by packed launches
// (each pass one launch over every running block) at one shared dt, and read
// out when their step count is done.  A block's cells never read another
// block's, so a case's result does not depend on what else is in the pool.
// ---------------------------------------------------------------------------

struct PoolSlot {
  int state = 0;  // 0 free, 1 admitted (filling), 2 running, 3 done
  int nx = 0, ny = 0, nz = 0;
  long long cv = 0, vol = 0;
  int steps_left = 0;
  int active = -1;   // its row in the running table
  int reactor = -1;  // a closed reactor's row in the reactor table (no block)
};

struct pgb_pool {
  unsigned long long uid = 0;
  unsigned version = 1;
  pgb_physics phys{};
  Species sp{};
  std::unique_ptr<Mech> mech;
  std::vector<pgb_stage> stages;
  int ne = 5;
  long long cap_cells = 0;
  int cap_blocks = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double *d_reg[MAXREGS] = {};
  double *d_met = nullptr, *d_state = nullptr, *d_tr = nullptr, *d_hsp = nullptr, *d_grads = nullptr;
  double *d_F[3] = {};
  double *d_dt = nullptr, *d_host = nullptr;  // dt, and the staging of one block's interior
  long long host_cap = 0;
  BlockDev *d_blks = nullptr;  // every slot's descriptor, by slot
  BlockDev *d_run = nullptr;   // the running table, by row
  HaloEntry *d_halo = nullptr;
  long long halo_cap = 0, nhalo = 0, nhalo_l0 = 0;
  // the same halo as boxes (k_halo_boxes): each running block's six face
  // halos, NG deep, periodic onto itself, and their CTA table
  HaloPatch *d_boxes = nullptr;
  int2 *d_boxcta = nullptr;
  long long box_cap = 0, boxcta_cap = 0, nboxcta = 0;
  // the first face layer's boxes (the gradients' fill): the last
  // 6 x blocks boxes of d_boxes, their CTA table after the full one's
  long long nboxcta0 = 0;
  int2 *d_ctab = nullptr;  // the running blocks' tile tables, one per range, end to end
  long long ctab_cap = 0, ctab_off[5] = {}, nctab[5] = {};
  // closed constant-volume reactors, a cell each: registers [component][rcap]
  // per register, each reactor's last T, the free rows, the running rows
  long long rcap = 0;
  double *d_rq[MAXREGS] = {};
  double *d_rT = nullptr;
  std::vector<int> rfree;
  std::vector<int> rrun;
  int *d_rrun = nullptr;
  // the fused passes take the blocks' stages (the case's batched form 2)
  bool fused = false;
  std::vector<PoolSlot> slots;
  std::map<long long, long long> free_;  // arena ranges: start -> cells
  std::vector<BlockDev> run;             // running blocks, host copy
  bool dirty = true;
  float last_ms = 0.0f;
  int last_launches = 0;
  // one step of the running set, captured; replayed until the set changes
  cudaGraphExec_t step_graph = nullptr;
  int step_graph_launches = 0;
};

namespace {

int pool_current(pgb_pool *p) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  Uploaded &u = g_plain_up[p->phys.ns - 1];
  // a pool's tables share the units' constant memory with the cases: keyed
  // by the pool's own unique id, handed over as a case's are
  if (!u.same(p->uid, p->version, dev)) {
    static MathTables mt;
    static bool filled = false;
    if (!filled) math_tables_fill(mt), filled = true;
    RET(take_tables(u, p->uid, p->version, dev, p->stream));
    RET(kPlain[p->phys.ns - 1].upload(&p->sp, p->mech.get(), p->mech ? &mt : nullptr, p->stream));
  }
  return PGB_OK;
}

// the slot's block as the kernels see it: halo NG deep, cells from cv
BlockDev slot_dev(const PoolSlot &s) {
  BlockDev D{};
  D.nx = s.nx, D.ny = s.ny, D.nz = s.nz;
  D.X = s.nx + 2 * NG, D.Y = s.ny + 2 * NG, D.Z = s.nz + 2 * NG;
  D.vol = s.vol;
  D.cv = s.cv;
  return D;
}

// the running table and its halo: each block periodic onto itself, the face
// halos NG deep, every block's first layer before any second layer
int pool_rebuild(pgb_pool *p) {
  p->run.clear();
  p->rrun.clear();
  for (size_t q = 0; q < p->slots.size(); q++) {
    PoolSlot &s = p->slots[q];
    s.active = -1;
    if (s.state != 2) continue;
    if (s.reactor >= 0) {
      p->rrun.push_back(s.reactor);
      continue;
    }
    s.active = (int)p->run.size();
    p->run.push_back(slot_dev(s));
  }
  // the boxes: for each running block and face, the NG halo planes, i
  // fastest, each cell's source n cells across along the face's axis
  // and, after them, the first layer alone (depth 1, next to the interior),
  // the gradients' fill; no per-cell list is built
  std::vector<HaloPatch> boxes;
  for (int depth : {NG, 1})
    for (const BlockDev &D : p->run) {
      const int n[3] = {D.nx, D.ny, D.nz};
      const int step[3] = {1, D.X, D.X * D.Y};
      for (int a = 0; a < 3; a++)
        for (int side = 0; side < 2; side++) {
          int lo[3] = {NG, NG, NG}, ext[3] = {n[0], n[1], n[2]};
          lo[a] = side == 0 ? NG - depth : NG + n[a];
          ext[a] = depth;
          HaloPatch P{};
          P.dcv = P.scv = D.cv;
          P.dvol = P.svol = (int)D.vol;
          P.d0 = (int)cell_index(D, lo[0], lo[1], lo[2]);
          P.s0 = P.d0 + (side == 0 ? 1 : -1) * n[a] * step[a];
          for (int d = 0; d < 3; d++) P.dst[d] = P.sst[d] = step[d];
          P.n0 = ext[0], P.n1 = ext[1], P.cells = ext[0] * ext[1] * ext[2];
          boxes.push_back(P);
        }
    }
  std::vector<int2> bcta;
  const int nfull = (int)boxes.size() / 2;
  for (int q = 0; q < (int)boxes.size(); q++) {
    if (q == nfull) p->nboxcta = (long long)bcta.size();
    for (int t = 0; t < (boxes[q].cells + 255) / 256; t++) bcta.push_back(make_int2(q, t));
  }
  if (boxes.empty()) p->nboxcta = 0;
  p->nboxcta0 = (long long)bcta.size() - p->nboxcta;
  if ((long long)boxes.size() > p->box_cap || (long long)bcta.size() > p->boxcta_cap) {
    CK(cudaStreamSynchronize(p->stream));
    if (p->d_boxes) CK(cudaFree(p->d_boxes));
    if (p->d_boxcta) CK(cudaFree(p->d_boxcta));
    p->d_boxes = nullptr, p->d_boxcta = nullptr;
    p->box_cap = std::max<long long>((long long)boxes.size(), 2 * p->box_cap);
    p->boxcta_cap = std::max<long long>((long long)bcta.size(), 2 * p->boxcta_cap);
    CK(cudaMalloc(&p->d_boxes, sizeof(HaloPatch) * std::max<long long>(1, p->box_cap)));
    CK(cudaMalloc(&p->d_boxcta, sizeof(int2) * std::max<long long>(1, p->boxcta_cap)));
  }
  if (!boxes.empty()) {
    CK(cudaMemcpyAsync(p->d_boxes, boxes.data(), sizeof(HaloPatch) * boxes.size(), cudaMemcpyHostToDevice, p->stream));
    CK(cudaMemcpyAsync(p->d_boxcta, bcta.data(), sizeof(int2) * bcta.size(), cudaMemcpyHostToDevice, p->stream));
  }
  p->nhalo_l0 = p->nhalo = 0;
  if (!p->run.empty())
    CK(cudaMemcpyAsync(p->d_run, p->run.data(), sizeof(BlockDev) * p->run.size(), cudaMemcpyHostToDevice, p->stream));
  if (!p->rrun.empty())
    CK(cudaMemcpyAsync(p->d_rrun, p->rrun.data(), sizeof(int) * p->rrun.size(), cudaMemcpyHostToDevice, p->stream));
  // each range's tiles: as many 256-thread CTAs as each block needs, no more
  std::vector<int2> tiles;
  for (int r = 0; r < 5; r++) {
    p->ctab_off[r] = (long long)tiles.size();
    for (int row = 0; row < (int)p->run.size(); row++) {
      const long long n = (range_size(p->run[row], r) + 255) / 256;
      for (long long t = 0; t < n; t++) tiles.push_back(make_int2(row, (int)t));
    }
    p->nctab[r] = (long long)tiles.size() - p->ctab_off[r];
  }
  if ((long long)tiles.size() > p->ctab_cap) {
    CK(cudaStreamSynchronize(p->stream));
    if (p->d_ctab) CK(cudaFree(p->d_ctab));
    p->d_ctab = nullptr;
    const long long cap = std::max<long long>((long long)tiles.size(), 2 * p->ctab_cap);
    CK(cudaMalloc(&p->d_ctab, sizeof(int2) * cap));
    p->ctab_cap = cap;
  }
  if (!tiles.empty())
    CK(cudaMemcpyAsync(p->d_ctab, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, p->stream));
  // the host vectors are read by the copies above: wait before they change
  CK(cudaStreamSynchronize(p->stream));
  p->dirty = false;
  return PGB_OK;
}

// one periodic block's face halos (NG deep) from its own interior, comps
// components: the copy the running table's halo makes, for a block not yet
// running
__global__ void k_selfhalo(const BlockDev *__restrict__ blks, int b, double *__restrict__ base, int comps) {
  const BlockDev &B = blks[b];
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= B.vol) return;
  const int i = (int)(t % B.X), j = (int)((t / B.X) % B.Y), k = (int)(t / ((long long)B.X * B.Y));
  const int oi = i < NG || i >= NG + B.nx, oj = j < NG || j >= NG + B.ny, ok = k < NG || k >= NG + B.nz;
  if (oi + oj + ok != 1) return;
  const int si = oi ? (i < NG ? i + B.nx : i - B.nx) : i;
  const int sj = oj ? (j < NG ? j + B.ny : j - B.ny) : j;
  const int sk = ok ? (k < NG ? k + B.nz : k - B.nz) : k;
  double *d = base + comps * B.cv;
  const long long dc = cell_index(B, i, j, k), sc = cell_index(B, si, sj, sk);
  for (int c = 0; c < comps; c++) d[c * B.vol + dc] = d[c * B.vol + sc];
}

PlainCase pool_plain(pgb_pool *p, const BlockDev *d_blks, const BlockDev *h_blks, int n) {
  PlainCase pc{};
  pc.d_blks = d_blks;
  pc.h_blks = h_blks;
  pc.nblocks = n;
  pc.state = p->d_state, pc.tr = p->d_tr, pc.hsp = p->d_hsp, pc.grads = p->d_grads;
  for (int a = 0; a < 3; a++) pc.F[a] = p->d_F[a];
  pc.met = p->d_met;
  pc.halo = p->d_halo;
  pc.nhalo = p->nhalo, pc.nhalo_l0 = p->nhalo_l0;
  // the boxes describe the running table's blocks, built with it
  if (d_blks == p->d_run) {
    pc.boxes = p->d_boxes, pc.boxcta = p->d_boxcta, pc.nboxcta = p->nboxcta;
    pc.boxes0 = p->d_boxes, pc.boxcta0 = p->d_boxcta + p->nboxcta, pc.nboxcta0 = p->nboxcta0;
  }
  pc.visc = sim_visc(p->phys.simulator);
  pc.primary = p->phys.primary, pc.recon = p->phys.recon, pc.limiter = p->phys.limiter;
  pc.chem = p->phys.chemistry == PGB_CHEM_COUPLED;
  pc.realgas = p->phys.eos == PGB_EOS_REALGAS || p->phys.eos == PGB_EOS_REALGAS_DF;
  pc.packed = 1;
  pc.dt = p->d_dt;
  // the pool's blocks are thin (a 1-D domain's halo is most of its cells)
  pc.rcell_inner = 1;
  pc.stream = p->stream;
  return pc;
}

// the running table's packing: its tile tables
void pool_tiles(const pgb_pool *p, PlainCase &pc) {
  for (int r = 0; r < 5; r++) {
    pc.ctab[r] = p->d_ctab ? p->d_ctab + p->ctab_off[r] : nullptr;
    pc.nctab[r] = p->nctab[r];
  }
}

void count_cb(void *ctx, int) { ++*(int *)ctx; }

int pool_slot(pgb_pool *p, int slot, int want) {
  if (!p) return fail(PGB_ERR_ARG, "null pool");
  if (slot < 0 || slot >= (int)p->slots.size() || p->slots[slot].state == 0) return fail(PGB_ERR_ARG, "no such slot");
  if (want >= 0 && p->slots[slot].state != want) return fail(PGB_ERR_STATE, "the slot is not in that state");
  return PGB_OK;
}

int pool_stage_host(pgb_pool *p, long long n) {
  if (n > p->host_cap) {
    // queued work may still read the old staging buffer
    CK(cudaStreamSynchronize(p->stream));
    if (p->d_host) CK(cudaFree(p->d_host));
    p->d_host = nullptr;
    CK(cudaMalloc(&p->d_host, sizeof(double) * n));
    p->host_cap = n;
  }
  return PGB_OK;
}

// one RK step of the running set's launches on the pool's stream: per stage
// the reactors' kernel, then the blocks' fused passes (or the right-hand side
// and the combines)
int pool_launch_step(pgb_pool *p, int &launches) {
  const int nrun = (int)p->run.size(), nreac = (int)p->rrun.size();
  PlainCase pc = pool_plain(p, p->d_run, p->run.data(), nrun);
  pool_tiles(p, pc);
  pc.mark = count_cb;
  pc.ctx = &launches;
  const dim3 g((unsigned)p->nctab[R_INNER], 1, 1);
  const int2 *inner_tiles = pc.ctab[R_INNER];
  // a stage's combines on a register table, in place: own first, dQ as
  // src -1, the first combine's value (already in the thread) as src -2
  auto combines = [&](const pgb_stage &st, double *const *reg, RCombine *out) {
    int written0 = -1;
    auto term = [&](RCombine &rc, int n, int r, double w) {
      const bool dq = r < 0 || r == st.dq;
      rc.src[n] = dq ? -1 : r == written0 ? -2 : 0;
      rc.X[n] = rc.src[n] < 0 ? nullptr : reg[r];
      rc.w[n] = w;
    };
    for (int m = 0; m < st.ncombine; m++) {
      const pgb_combine &cb = st.combine[m];
      RCombine &rc = out[m];
      rc = RCombine{};
      rc.out = reg[cb.out];
      rc.step = cb.step;
      rc.write = 1;
      int n = 0;
      if (cb.own) term(rc, n++, cb.out, cb.wout);
      for (int q = 0; q < cb.nterms; q++) term(rc, n++, cb.reg[q], cb.w[q]);
      rc.nterms = n;
      if (m == 0) written0 = cb.out;
    }
  };
  for (const pgb_stage &st : p->stages) {
    if (nreac) {
      ReactorStage rs{};
      rs.Q = p->d_rq[st.q];
      rs.T = p->d_rT;
      rs.rows = p->d_rrun;
      rs.n = nreac;
      rs.cap = p->rcap;
      rs.dt = p->d_dt;
      rs.ncomb = st.ncombine;
      combines(st, p->d_rq, rs.comb);
      RET(kPlain[p->phys.ns - 1].reactors(&rs, p->stream));
      launches++;
    }
    if (nrun == 0) continue;
    if (p->fused) {
      // the fused passes: the divergence and the combines in one pass
      RStage r{};
      r.Q = p->d_reg[st.q];
      r.dQ = p->d_reg[st.dq];
      r.ncomb = st.ncombine;
      combines(st, p->d_reg, r.comb);
      RET(kPlain[p->phys.ns - 1].fused(&pc, &r));
      continue;
    }
    RET(kPlain[p->phys.ns - 1].rhs(&pc, p->d_reg[st.q], p->d_reg[st.dq]));
    for (int m = 0; m < st.ncombine; m++) {
      const pgb_combine &cb = st.combine[m];
      CombineDev cd{};
      cd.out = p->d_reg[cb.out];
      cd.own = cb.own;
      cd.wout = cb.wout;
      cd.nterms = cb.nterms;
      cd.step = cb.step;
      for (int n = 0; n < cb.nterms; n++) {
        cd.X[n] = p->d_reg[cb.reg[n] < 0 ? st.dq : cb.reg[n]];
        cd.w[n] = cb.w[n];
      }
      k_combine<<<g, 256, 0, p->stream>>>(p->d_run, 0, p->ne, cd, p->d_dt, inner_tiles);
      launches++;
    }
  }
  CK(cudaGetLastError());
  return PGB_OK;
}

}  // namespace

extern "C" {

int pgb_pool_create(const pgb_case *proto, long long max_cells, int max_blocks, pgb_pool **out) {
  if (!proto || !out) return fail(PGB_ERR_ARG, "null argument");
  if (!proto->finalized) return fail(PGB_ERR_STATE, "finalize the prototype case first");
  if (sim_df(proto->phys.simulator)) return fail(PGB_ERR_UNSUPPORTED, "the pool does not take the double flux");
  if (proto->phys.chemistry == PGB_CHEM_SUBSTEPPED)
    return fail(PGB_ERR_UNSUPPORTED, "the pool takes the coupled chemistry, not the sub-stepped");
  if (max_cells < 64 || max_blocks < 1 || max_blocks > 65535)
    return fail(PGB_ERR_ARG, "a pool holds at least 64 cells and 1 to 65535 blocks");
  auto p = std::make_unique<pgb_pool>();
  p->uid = ++g_next_uid;
  p->phys = proto->phys;
  p->sp = proto->sp;
  if (proto->mech) p->mech = std::make_unique<Mech>(*proto->mech);
  p->stages = proto->stages;
  p->ne = proto->ne;
  p->cap_cells = max_cells;
  p->cap_blocks = max_blocks;
  p->slots.resize(max_blocks);
  p->free_[0] = max_cells;
  const int ns = p->phys.ns, ne = p->ne;
  const size_t n = (size_t)max_cells;
  CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&p->ev0));
  CK(cudaEventCreate(&p->ev1));
  for (int r = 0; r < p->phys.nregs; r++) CK(cudaMalloc(&p->d_reg[r], sizeof(double) * ne * n));
  CK(cudaMalloc(&p->d_met, sizeof(double) * M_NCOMP * n));
  CK(cudaMalloc(&p->d_state, sizeof(double) * SW * n));
  CK(cudaMalloc(&p->d_tr, sizeof(double) * (2 + ns) * n));
  CK(cudaMalloc(&p->d_hsp, sizeof(double) * ns * n));
  CK(cudaMalloc(&p->d_grads, sizeof(double) * 3 * (ne - 1) * n));
  for (int a = 0; a < 3; a++) CK(cudaMalloc(&p->d_F[a], sizeof(double) * ne * n));
  CK(cudaMalloc(&p->d_dt, sizeof(double)));
  CK(cudaMalloc(&p->d_blks, sizeof(BlockDev) * max_blocks));
  CK(cudaMalloc(&p->d_run, sizeof(BlockDev) * max_blocks));
  // a closed reactor a slot at most
  p->rcap = max_blocks;
  for (int r = 0; r < p->phys.nregs; r++) {
    CK(cudaMalloc(&p->d_rq[r], sizeof(double) * ne * p->rcap));
    CK(cudaMemsetAsync(p->d_rq[r], 0, sizeof(double) * ne * p->rcap, p->stream));
  }
  CK(cudaMalloc(&p->d_rT, sizeof(double) * p->rcap));
  CK(cudaMalloc(&p->d_rrun, sizeof(int) * p->rcap));
  for (int r = (int)p->rcap - 1; r >= 0; r--) p->rfree.push_back(r);
  // the blocks step on the fused passes where the physics takes them: the
  // ideal gases (every pool block is periodic onto itself, of two cells or
  // more per axis, so neither a boundary nor a block's size bars them)
  p->fused = (p->phys.simulator == PGB_EULER || p->phys.simulator == PGB_NAVIER_STOKES) &&
             (p->phys.eos == PGB_EOS_CPG || p->phys.eos == PGB_EOS_TPG);
  *out = p.release();
  return PGB_OK;
}

int pgb_pool_destroy(pgb_pool *p) {
  if (!p) return PGB_OK;
  if (p->stream) cudaStreamSynchronize(p->stream);
  for (auto &r : p->d_reg)
    if (r) cudaFree(r);
  for (auto &r : p->d_rq)
    if (r) cudaFree(r);
  void *ptrs[] = {p->d_met, p->d_state, p->d_tr, p->d_hsp, p->d_grads, p->d_F[0], p->d_F[1], p->d_F[2],
                  p->d_dt, p->d_host, p->d_blks, p->d_run, p->d_halo, p->d_ctab, p->d_rT, p->d_rrun, p->d_boxes, p->d_boxcta};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (p->step_graph) cudaGraphExecDestroy(p->step_graph);
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  if (p->stream) forget_stream(p->stream), cudaStreamDestroy(p->stream);
  delete p;
  return PGB_OK;
}

// a slot for an ni x nj x nk periodic block; PGB_ERR_NOMEM when the arena or
// the slot table has no room (the caller queues the case and tries later)
int pgb_pool_admit(pgb_pool *p, int ni, int nj, int nk, int *slot) {
  if (!p || !slot) return fail(PGB_ERR_ARG, "null argument");
  if (ni < 2 || nj < 2 || nk < 2 || ni > 30000 || nj > 30000 || nk > 30000)
    return fail(PGB_ERR_ARG, "a block has 2 to 30000 cells per axis");
  const long long vol = (long long)(ni + 2 * NG) * (nj + 2 * NG) * (nk + 2 * NG);
  int id = -1;
  for (int q = 0; q < (int)p->slots.size(); q++)
    if (p->slots[q].state == 0) {
      id = q;
      break;
    }
  if (id < 0) return fail(PGB_ERR_NOMEM, "every slot of the pool is taken");
  // first fit over the arena's free ranges
  auto it = p->free_.begin();
  for (; it != p->free_.end(); ++it)
    if (it->second >= vol) break;
  if (it == p->free_.end()) return fail(PGB_ERR_NOMEM, "the pool's arena has no free range that large");
  const long long cv = it->first, left = it->second - vol;
  p->free_.erase(it);
  if (left > 0) p->free_[cv + vol] = left;
  PoolSlot &s = p->slots[id];
  s = PoolSlot{};
  s.state = 1;
  s.nx = ni, s.ny = nj, s.nz = nk;
  s.cv = cv, s.vol = vol;
  const BlockDev D = slot_dev(s);
  // a new occupant starts from zeros: its halo's first Newton from the cold
  // guess, whatever the range held before
  for (int r = 0; r < p->phys.nregs; r++)
    CK(cudaMemsetAsync(p->d_reg[r] + (size_t)p->ne * cv, 0, sizeof(double) * p->ne * vol, p->stream));
  CK(cudaMemsetAsync(p->d_state + (size_t)SW * cv, 0, sizeof(double) * SW * vol, p->stream));
  // from pageable memory: the call returns once D is staged, so the stack copy may go
  CK(cudaMemcpyAsync(p->d_blks + id, &D, sizeof(BlockDev), cudaMemcpyHostToDevice, p->stream));
  *slot = id;
  return PGB_OK;
}

// a slot for a closed constant-volume reactor: a cell, no grid
int pgb_pool_admit_reactor(pgb_pool *p, int *slot) {
  if (!p || !slot) return fail(PGB_ERR_ARG, "null argument");
  if (p->phys.chemistry != PGB_CHEM_COUPLED) return fail(PGB_ERR_UNSUPPORTED, "a reactor takes the coupled chemistry");
  if (p->phys.eos != PGB_EOS_TPG) return fail(PGB_ERR_UNSUPPORTED, "a reactor takes the thermally perfect gas");
  int id = -1;
  for (int q = 0; q < (int)p->slots.size(); q++)
    if (p->slots[q].state == 0) {
      id = q;
      break;
    }
  if (id < 0 || p->rfree.empty()) return fail(PGB_ERR_NOMEM, "every slot of the pool is taken");
  PoolSlot &s = p->slots[id];
  s = PoolSlot{};
  s.state = 1;
  s.nx = s.ny = s.nz = 1;
  s.reactor = p->rfree.back();
  p->rfree.pop_back();
  *slot = id;
  return PGB_OK;
}

// a slot's metric array, laid out as pgb_metric_set's
int pgb_pool_metric_set(pgb_pool *p, int slot, int which, const double *host, long count) {
  RET(pool_slot(p, slot, 1));
  if (p->slots[slot].reactor >= 0) return fail(PGB_ERR_ARG, "a reactor has no grid");
  if (!host || which < 0 || which >= PGB_NMETRICS) return fail(PGB_ERR_ARG, "no such metric");
  const BlockDev D = slot_dev(p->slots[slot]);
  static const int comps[PGB_NMETRICS] = {3, 1, 9, 3, 3, 3, 3, 3, 3};
  static const int first[PGB_NMETRICS] = {M_XCC, M_DETJINV, M_JINV, M_S, M_S + 3, M_S + 6, M_XF, M_XF + 3, M_XF + 6};
  const int face = which >= PGB_ARR_IS ? (which - PGB_ARR_IS) % 3 : -1;
  const int X = D.X + (face == 0), Y = D.Y + (face == 1), Z = D.Z + (face == 2);
  const int nc = comps[which];
  if (count != (long)X * Y * Z * nc) return fail(PGB_ERR_ARG, "metric array of the wrong size");
  // the host array is F order over its own extents, as the device's: a cell
  // array copies straight; a face array's rows (i faces), planes (j) or
  // volumes (k) are one cell longer, and that last cell, past the halo, is
  // never read: a pitched copy drops it
  double *dst = p->d_met + (size_t)M_NCOMP * D.cv + (size_t)first[which] * D.vol;
  const size_t w = sizeof(double);
  if (face < 0)
    CK(cudaMemcpyAsync(dst, host, w * nc * D.vol, cudaMemcpyHostToDevice, p->stream));
  else if (face == 0)
    CK(cudaMemcpy2DAsync(dst, w * D.X, host, w * X, w * D.X, (size_t)D.Y * D.Z * nc, cudaMemcpyHostToDevice, p->stream));
  else if (face == 1)
    CK(cudaMemcpy2DAsync(dst, w * D.X * D.Y, host, w * D.X * Y, w * D.X * D.Y, (size_t)D.Z * nc,
                         cudaMemcpyHostToDevice, p->stream));
  else
    CK(cudaMemcpy2DAsync(dst, w * D.vol, host, w * (size_t)D.X * D.Y * Z, w * D.vol, (size_t)nc,
                         cudaMemcpyHostToDevice, p->stream));
  // pageable source: each copy has taken the host data when it returns, and
  // the launches that read it follow on the same stream
  return PGB_OK;
}

// a slot's Q and state from interior primitives (F order, as pgb_set_prims)
int pgb_pool_set_prims(pgb_pool *p, int slot, const double *host, long count) {
  RET(pool_slot(p, slot, 1));
  const PoolSlot &s = p->slots[slot];
  if (!host || count != (long)s.nx * s.ny * s.nz * p->ne) return fail(PGB_ERR_ARG, "primitives of the wrong size");
  RET(pool_current(p));
  RET(pool_stage_host(p, count));
  CK(cudaMemcpyAsync(p->d_host, host, sizeof(double) * count, cudaMemcpyHostToDevice, p->stream));
  if (s.reactor >= 0)
    return kPlain[p->phys.ns - 1].reactor_prims(p->d_host, p->d_rq[0], p->d_rT, s.reactor, p->rcap, p->stream);
  // the unit reads the launch size from the host table at the slot's index
  std::vector<BlockDev> hb((size_t)slot + 1);
  hb[slot] = slot_dev(s);
  const PlainCase pc = pool_plain(p, p->d_blks, hb.data(), slot + 1);
  RET(kPlain[p->phys.ns - 1].fromprims(&pc, slot, p->d_host, p->d_reg[0]));
  // a halo cell's first Newton starts from the stored T of the cell it copies
  k_selfhalo<<<grid_for(hb[slot].vol, 256), 256, 0, p->stream>>>(p->d_blks, slot, p->d_state, SW);
  CK(cudaGetLastError());
  return PGB_OK;
}

// the slot joins the running cases at the next step, for nsteps steps
int pgb_pool_start(pgb_pool *p, int slot, int nsteps) {
  RET(pool_slot(p, slot, 1));
  if (nsteps < 1) return fail(PGB_ERR_ARG, "at least one step");
  p->slots[slot].state = 2;
  p->slots[slot].steps_left = nsteps;
  p->dirty = true;
  return PGB_OK;
}

// nsteps RK steps of every running case at dt; a case whose count runs out
// is done and leaves the running set after that step.  A step's launches
// depend on the running set alone (dt is read on the device), so the step is
// captured once per set and replayed until an admission, a release or a case
// finishing changes it.
int pgb_pool_step(pgb_pool *p, double dt, int nsteps) {
  if (!p) return fail(PGB_ERR_ARG, "null pool");
  if (nsteps < 1) return fail(PGB_ERR_ARG, "at least one step");
  RET(pool_current(p));
  k_setscalar<<<1, 1, 0, p->stream>>>(p->d_dt, dt);
  int launches = 0;
  CK(cudaEventRecord(p->ev0, p->stream));
  for (int it = 0; it < nsteps; it++) {
    if (p->dirty) {
      RET(pool_rebuild(p));
      if (p->step_graph) cudaGraphExecDestroy(p->step_graph);
      p->step_graph = nullptr;
    }
    if (p->run.empty() && p->rrun.empty()) break;
    if (!p->step_graph) {
      int n = 0;
      CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = pool_launch_step(p, n);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(p->stream, &g);
      if (rc != PGB_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc != PGB_OK ? rc : fail(PGB_ERR_CUDA, std::string("pool step capture: ") + cudaGetErrorString(e));
      }
      const cudaError_t ei = cudaGraphInstantiate(&p->step_graph, g, 0);
      cudaGraphDestroy(g);
      CK(ei);
      p->step_graph_launches = n;
    }
    CK(cudaGraphLaunch(p->step_graph, p->stream));
    launches += p->step_graph_launches;
    for (auto &s : p->slots)
      if (s.state == 2 && --s.steps_left == 0) s.state = 3, p->dirty = true;
  }
  CK(cudaEventRecord(p->ev1, p->stream));
  CK(cudaEventSynchronize(p->ev1));
  CK(cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1));
  p->last_launches = launches;
  return PGB_OK;
}

// the done slots, up to cap of them; n the count there are
int pgb_pool_done(const pgb_pool *p, int *slots, int cap, int *n) {
  if (!p || !n || (cap > 0 && !slots)) return fail(PGB_ERR_ARG, "null argument");
  int k = 0;
  for (int q = 0; q < (int)p->slots.size(); q++)
    if (p->slots[q].state == 3) {
      if (k < cap) slots[k] = q;
      k++;
    }
  *n = k;
  return PGB_OK;
}

// a slot's register reg over its interior, F order (as pgb_array_get)
int pgb_pool_get(pgb_pool *p, int slot, int reg, double *host, long count) {
  RET(pool_slot(p, slot, -1));
  const PoolSlot &s = p->slots[slot];
  if (reg < 0 || reg >= p->phys.nregs) return fail(PGB_ERR_ARG, "no such register");
  if (!host || count != (long)s.nx * s.ny * s.nz * p->ne) return fail(PGB_ERR_ARG, "host array of the wrong size");
  if (s.reactor >= 0) {
    // the reactor's column of the [component][capacity] table
    CK(cudaMemcpy2DAsync(host, sizeof(double), p->d_rq[reg] + s.reactor, sizeof(double) * p->rcap, sizeof(double),
                         (size_t)p->ne, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    return PGB_OK;
  }
  RET(pool_stage_host(p, count));
  k_pack<<<grid_for((long long)s.nx * s.ny * s.nz, 256), 256, 0, p->stream>>>(p->d_blks, slot, p->ne, p->d_reg[reg],
                                                                               p->d_host);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, p->d_host, sizeof(double) * count, cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return PGB_OK;
}

// the slot and its arena range are free again
int pgb_pool_release(pgb_pool *p, int slot) {
  RET(pool_slot(p, slot, -1));
  PoolSlot &s = p->slots[slot];
  if (s.state == 2) p->dirty = true;
  if (s.reactor >= 0) {
    p->rfree.push_back(s.reactor);
    s = PoolSlot{};
    return PGB_OK;
  }
  // give the range back, merged with free neighbours
  long long cv = s.cv, vol = s.vol;
  auto nx = p->free_.lower_bound(cv);
  if (nx != p->free_.end() && nx->first == cv + vol) {
    vol += nx->second;
    p->free_.erase(nx);
  }
  auto pv = p->free_.lower_bound(cv);
  if (pv != p->free_.begin()) {
    --pv;
    if (pv->first + pv->second == cv) {
      cv = pv->first;
      vol += pv->second;
      p->free_.erase(pv);
    }
  }
  p->free_[cv] = vol;
  s = PoolSlot{};
  return PGB_OK;
}

// the largest free range of cells (halo included), and the running and done counts
int pgb_pool_info(const pgb_pool *p, long long *largest_free, int *running, int *done) {
  if (!p) return fail(PGB_ERR_ARG, "null pool");
  long long big = 0;
  for (auto &f : p->free_) big = std::max(big, f.second);
  int r = 0, d = 0;
  for (auto &s : p->slots) r += s.state == 2, d += s.state == 3;
  if (largest_free) *largest_free = big;
  if (running) *running = r;
  if (done) *done = d;
  return PGB_OK;
}

// the last pgb_pool_step's device time and its launches
int pgb_pool_last(const pgb_pool *p, float *ms, int *launches) {
  if (!p) return fail(PGB_ERR_ARG, "null pool");
  if (ms) *ms = p->last_ms;
  if (launches) *launches = p->last_launches;
  return PGB_OK;
}

}  // extern "C"
