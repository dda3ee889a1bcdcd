/*
 * pgb200: PEREGRINE's right-hand side and Runge-Kutta stage on one B200.
 *
 * A plain C ABI: opaque handles, plain pointers and sizes, an int status on
 * every call (0 = success), and the text of the last failure on the calling
 * thread from pgb_last_error().  Nothing here names a torch or CUDA type; a
 * CUDA stream crosses as a void pointer.
 *
 * What each entry replaces in the reference (paths inside kaschau/Peregrine):
 *
 *  - The reference renders every kernel per case into a C++ unit and calls its
 *    extern "C" pg_<symbol>(const K, const pg::Tiling) entry through the CUDA
 *    driver (peregrine/backend/device/kernels/launch.mako:5-12,
 *    peregrine/backend/device/backend.py:33-48).  Here the kernels are compiled
 *    once for sm_100a and selected by the case description.
 *  - The solver-level calls (peregrine/multiblock/solver.py:246-364: rhs,
 *    advance, step, set_prims, the arrays' get/set) map onto pgb_rhs,
 *    pgb_step, pgb_set_prims, pgb_array_set and pgb_array_get.
 */
#ifndef PGB200_H
#define PGB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; a CUDA runtime failure is PGB_ERR_CUDA with its text in
 * pgb_last_error() (the reference maps driver codes to typed exceptions,
 * peregrine/backend/cuda/driver.py:7-55) */
enum {
  PGB_OK = 0,
  PGB_ERR_ARG = 1,       /* a bad argument: a size, a name, an index */
  PGB_ERR_STATE = 2,     /* a call out of order: e.g. a step before finalize */
  PGB_ERR_CUDA = 3,      /* a CUDA runtime error */
  PGB_ERR_NOMEM = 4,     /* a device allocation refused */
  PGB_ERR_UNSUPPORTED = 5, /* a physics choice this build does not have */
  PGB_ERR_TIMEOUT = 6,   /* a bounded device wait gave up (status word set) */
};

/* physics selectors: the config's names (peregrine/config.py:12-98) */
/* the double flux's simulators freeze the real gas's tangent plane each step
 * (peregrine/simulator/eulerdf/simulator.py, navstokesdf/simulator.py) */
enum { PGB_EULER = 0, PGB_NAVIER_STOKES = 1, PGB_EULER_DF = 2, PGB_NAVIER_STOKES_DF = 3 };
enum { PGB_EOS_CPG = 0, PGB_EOS_TPG = 1, PGB_EOS_REALGAS = 2, PGB_EOS_REALGAS_DF = 3 };
enum { PGB_FLUX_KEPAEC = 0, PGB_FLUX_HLLC = 1, PGB_FLUX_RUSANOV = 2, PGB_FLUX_AUSMUP = 3 };
enum { PGB_RECON_CONSTANT = 0, PGB_RECON_MUSCL = 1 };
enum { PGB_TRANS_NONE = 0, PGB_TRANS_CONSTANT = 1, PGB_TRANS_KINETIC = 2 };
/* chemistry: none, finite-rate coupled into the right-hand side
 * (peregrine/simulator/chemint/coupled.py), or sub-stepped over the step with
 * stiff-cell compaction (peregrine/simulator/chemint/substepped.py) */
enum { PGB_CHEM_NONE = 0, PGB_CHEM_COUPLED = 1, PGB_CHEM_SUBSTEPPED = 2 };
/* the launch paths */
/* the launch paths: the batched fused kernel; the per-block kernels one
 * launch per block and pass (the reference's order); the same kernels
 * packed, each pass one launch over every block */
enum { PGB_PATH_BATCHED = 0, PGB_PATH_PER_BLOCK = 1, PGB_PATH_PACKED = 2 };

/* the per-cell and per-face arrays of a block the caller sets (metrics) or
 * reads and writes (registers, prims): the reference's array names
 * (peregrine/multiblock/block/grid.py:123-202) */
enum {
  PGB_ARR_XCC = 0,     /* cell centres, 3 */
  PGB_ARR_DETJINV = 1, /* 1 / volume, 1 */
  PGB_ARR_JINV = 2,    /* inverse Jacobian, 3 x 3 */
  PGB_ARR_IS = 3, PGB_ARR_JS = 4, PGB_ARR_KS = 5,    /* face area vectors, 3 */
  PGB_ARR_IXC = 6, PGB_ARR_JXC = 7, PGB_ARR_KXC = 8, /* face centres, 3 */
  PGB_NMETRICS = 9
};

typedef struct pgb_case pgb_case;

typedef struct {
  int simulator;  /* PGB_EULER, PGB_NAVIER_STOKES, PGB_EULER_DF, PGB_NAVIER_STOKES_DF */
  int eos;        /* PGB_EOS_* */
  int primary;    /* PGB_FLUX_* */
  int recon;      /* PGB_RECON_* */
  int limiter;    /* with PGB_RECON_MUSCL: 1 koren, 2 minmod, 3 mc, 4 superbee, 5 vanleer */
  int trans;      /* PGB_TRANS_* */
  int ns;         /* species, >= 1 */
  int nregs;      /* Runge-Kutta registers the integrator needs, dQ included */
  double alpha;   /* alpha-damping coefficient */
  int chemistry;  /* PGB_CHEM_* */
} pgb_physics;

/* A finite-rate mechanism: the columns the reference's FiniteRateModel
 * works out (peregrine/simulator/mixture/chemistry/finiterate.py:29-51,
 * 122-160), one struct per reaction.  Species are numbered as the mixture's;
 * a side lists its species with nonzero coefficients. */
enum { PGB_RXN_ELEMENTARY = 0, PGB_RXN_THREEBODY = 1, PGB_RXN_LINDEMANN = 2, PGB_RXN_TROE = 3 };
#define PGB_MAXSIDE 4
#define PGB_MAXNET 8
typedef struct {
  int kind;        /* PGB_RXN_* */
  int reversible;
  int product;     /* 1: the product form, 0: the log form (finiterate.py:62-102) */
  int tb;          /* third-body set, -1 for none */
  int troe;        /* row of the Troe centre fit */
  int nfcent;      /* terms of the Troe centre; 0 floors it */
  int nfwd, nreact, nprod, nnet;
  int fwdsp[PGB_MAXSIDE], reactsp[PGB_MAXSIDE], prodsp[PGB_MAXSIDE], netsp[PGB_MAXNET];
  double fwdorder[PGB_MAXSIDE], reactnu[PGB_MAXSIDE], prodnu[PGB_MAXSIDE];
  double netnu[PGB_MAXNET], netnuMW[PGB_MAXNET];
  double logA, b, EaR;        /* ln k = logA + b ln T - EaR / T */
  double logprA, prb, prEaR;  /* the falloff's pressure ratio, the same form */
  double nusum;               /* the net stoichiometry's sum */
} pgb_reaction;
typedef struct {
  double defeff;    /* default efficiency */
  int neff;
  int effsp[12];    /* species whose efficiency differs, and by how much */
  double effdev[12];
} pgb_thirdbody;
typedef struct {
  int nr, ntb, ntroe, nlfc, ng;
  const pgb_reaction *rxn;   /* [nr] */
  const pgb_thirdbody *tb;   /* [ntb] */
  const double *lfcpoly;     /* [ntroe][nlfc]: Troe's log10 centre in (ln T - troeuc) troeuhinv */
  const double *gpoly;       /* [ns][ng]: g / Ru T in ln T, less h298 / T (the "h298" table) */
  double logprefRu, prefRu, Rupref, logcfloor, maxgain, troeuc, troeuhinv;
} pgb_mechanism;

/* One Runge-Kutta combine: out = [wout out +] sum_n w[n] X[n], dt multiplying
 * the last term when step is set (peregrine/integrators/kernels/combine.mako).
 * A term whose reg is -1 is the stage's right-hand side dQ.  Registers are
 * logical (0 .. nregs-1 as the integrator names them). */
typedef struct {
  int out;
  int own;        /* 1: wout * out is the first term */
  double wout;
  int nterms;     /* 1 .. 3 */
  int reg[3];
  double w[3];
  int step;
} pgb_combine;

/* One stage: the register its right-hand side reads, the combines after it,
 * and the stage's time as a fraction of dt past the step's start, the clock
 * its boundary values read (peregrine/integrators/rungekutta.py:28-39) */
typedef struct {
  int q;
  int dq;         /* the logical register holding dQ on the per-block path */
  int ncombine;   /* 1 or 2 */
  pgb_combine combine[2];
  double tfrac;
} pgb_stage;

/* Boundary kinds: the reference's bcvals kinds
 * (peregrine/simulator/euler/bcs.py, peregrine/simulator/navstokes/bcs.py).
 * The values an entry gives, in order (each a program, below):
 *   SLIP_ADIA_WALL, NOSLIP_ADIA_WALL, SUP_OUT_FN: none
 *   SLIP_ISOT_WALL, NOSLIP_ISOT_WALL: T      MOV_ADIA_WALL: u v w
 *   MOV_ISOT_WALL: u v w T                    SUB_OUT_FP: p
 *   SUB_IN_FVT: u v w T, Y[ns - 1]            SUP_IN_FA: p u v w T, Y[ns - 1]
 *   SUB_IN_FTPTT: pt Tt, Y[ns - 1]            SUB_IN_FMT: mflux T, Y[ns - 1]
 * The no-slip and moving walls are the Navier-Stokes simulator's. */
enum {
  PGB_BC_SLIP_ADIA_WALL = 1,   /* slp-adia-wall */
  PGB_BC_SLIP_ISOT_WALL = 2,   /* slp-isot-wall */
  PGB_BC_NOSLIP_ADIA_WALL = 3, /* no-slp-adia-wall */
  PGB_BC_MOV_ADIA_WALL = 4,    /* mov-adia-wall */
  PGB_BC_NOSLIP_ISOT_WALL = 5, /* no-slp-isot-wall */
  PGB_BC_MOV_ISOT_WALL = 6,    /* mov-isot-wall */
  PGB_BC_SUB_IN_FVT = 7,       /* sub-in-fvt */
  PGB_BC_SUP_IN_FA = 8,        /* sup-in-fa */
  PGB_BC_SUB_IN_FTPTT = 9,     /* sub-in-ftptt */
  PGB_BC_SUB_IN_FMT = 10,      /* sub-in-fmt */
  PGB_BC_SUB_OUT_FP = 11,      /* sub-out-fp */
  PGB_BC_SUP_OUT_FN = 12,      /* sup-out-fn */
  PGB_BC_NKINDS = 13
};

/* A boundary value is a program for a small stack machine, evaluated at each
 * boundary face's centre (x, y, z) and the stage's time t: the reference's
 * expressions of x, y, z and t (peregrine/simulator/bcs.py:101-143) in
 * postfix.  CONST pushes its argument; X Y Z T push the coordinate or time;
 * the binary operations pop b then a and push a op b; the functions pop
 * their arguments the same way.  A program leaves one value and never holds
 * more than PGB_BC_STACK. */
enum {
  PGB_OP_CONST = 0, PGB_OP_X, PGB_OP_Y, PGB_OP_Z, PGB_OP_T,
  PGB_OP_ADD, PGB_OP_SUB, PGB_OP_MUL, PGB_OP_DIV, PGB_OP_NEG, PGB_OP_POW,
  PGB_OP_SIN, PGB_OP_COS, PGB_OP_TAN, PGB_OP_EXP, PGB_OP_LOG, PGB_OP_SQRT, PGB_OP_TANH,
  PGB_OP_ABS, PGB_OP_MIN, PGB_OP_MAX,
  PGB_NOPS
};
#define PGB_BC_STACK 16
#define PGB_BC_MAXOPS 4096

/* library */
const char *pgb_last_error(void);
int pgb_version(void);
int pgb_device_init(int ordinal);
int pgb_device_count(int *count);
int pgb_device_sync(void);
/* a device's free and total memory, bytes */
int pgb_mem_info(size_t *free_bytes, size_t *total_bytes);

/* a case: physics, species tables, blocks, connectivity, then finalize */
int pgb_case_create(const pgb_physics *phys, pgb_case **out);
int pgb_case_destroy(pgb_case *c);
/* a named species table of n doubles (names as the reference's mixture
 * constants: "Rsp", "cp0", "h298R", "MWinv", "hpoly0", "h298", "mu0",
 * "kappa0", "MWqinv", "wilkepair", "lewis") */
int pgb_case_set_table(pgb_case *c, const char *name, const double *values, long n);
/* the thermally perfect gas reads "cppolyR" (cp in ln T times R_sp) and
 * "hpoly" (h / R T), kinetic-theory transport "mupoly" and "kappapoly", each
 * [ns][terms] with 1 to 8 terms (peregrine/simulator/mixture/eos/tpg/model.py,
 * peregrine/simulator/mixture/transport/kinetic.py); the real gas those of
 * the thermally perfect gas and the cubic's: "cubicu", "cubicw",
 * "cubicsigma", "cubiceps" (one value each), "cubicsqrtac", "cubicb",
 * "cubicda", "cubicmTc", "cubiconepm", "vshift", "cubicsqrtacMW", "cubicbMW",
 * "cubicdaMW", "vshiftMW" (ns each; peregrine/simulator/mixture/eos/realgas/model.py:43-98) */
/* the case's finite-rate mechanism, copied; before finalize */
int pgb_case_set_mechanism(pgb_case *c, const pgb_mechanism *m);
/* The coupled chemistry's source kernel generated for the case's mechanism:
 * every reaction straight-line code with its species indices and constants as
 * literals, compiled for the device at pgb_case_finalize (NVRTC), as the
 * reference renders its finite-rate kernels
 * (peregrine/simulator/mixture/chemistry/kernels/finiterate.mako).  On by
 * default; off (before finalize) keeps the table-driven kernel, which walks
 * the mechanism's columns at run time.  Where NVRTC cannot be opened the
 * table-driven kernel stays in use; pgb_case_generated_chemistry says which
 * runs and, when it is not the generated one, why (up to cap bytes). */
int pgb_case_set_generated_chemistry(pgb_case *c, int on);
int pgb_case_generated_chemistry(const pgb_case *c, int *on, char *why, long long cap);
/* The generated source itself (len its length, up to cap bytes written), and
 * its compilation for sm_100a with nothing loaded (the compiler's log on
 * failure): host computations, before or after finalize. */
int pgb_case_rates_source(pgb_case *c, char *buf, long long cap, long long *len);
int pgb_case_rates_compile(pgb_case *c, char *log, long long cap);
/* the sub-stepped chemistry's options (the reference's chem-integration
 * section, peregrine/simulator/chemint/substepped.py:14-33): max-substeps
 * cap >= 1, bulk-substeps 1 <= bulk <= cap (bulk < cap compacts the stiff
 * cells into a second pass), stiff-bins 1..16, equilibrium-tolerance
 * 0 <= eqtol < 1 (0: no exit).  Defaults 200, 1, 8, 1e-7.  Before finalize. */
int pgb_case_set_substeps(pgb_case *c, int cap, int bulk, int bins, double eqtol);
/* each interior cell's substep count at the last right-hand side (host F
 * order, count = the block's interior cells), and the stiff list's header:
 * head[0] the cells listed, head[1 + b] bin b's, n = bins + 1 */
int pgb_substeps_get(pgb_case *c, int blk, int *host, long count);
int pgb_stiff_head(pgb_case *c, unsigned int *head, int n);
/* net production rates omega[n][ns], kg / m^3 / s, of n states rho[n],
 * Y[n][ns] (every species) and T[n], host arrays, by the device fold */
int pgb_production(pgb_case *c, long n, const double *rho, const double *Y, const double *T, double *omega);
/* a block of ni x nj x nk cells; its number is the order of the calls */
int pgb_case_add_block(pgb_case *c, int ni, int nj, int nk, int *blk);
/* face nface (1..6: i-low, i-high, j-low, j-high, k-low, k-high) of blk joins
 * face nbrface of nbr, orientation "123" (the lattice meshers' only one,
 * peregrine/mesher/base.py:117-133); nbr -1 is a boundary */
int pgb_case_connect(pgb_case *c, int blk, int nface, int nbr, int nbrface);
/* A boundary entry (one entry of the reference's bcvals,
 * peregrine/simulator/bcs.py:10-98): its kind (PGB_BC_*) and its values, value
 * v the program ops[starts[v] .. starts[v + 1]) with args the CONST operands
 * (one per op, read for CONST alone).  nvalues is what the kind reads for the
 * case's species.  Before finalize; *id numbers the entry. */
int pgb_case_add_bc(pgb_case *c, int kind, const int *ops, const double *args, const int *starts, int nvalues,
                    int *id);
/* A boundary face (connected with nbr -1) takes entry bc: the reference's
 * interface named in bcvals (peregrine/multiblock/solver.py:157-173).  A
 * boundary face given no entry keeps its halo as set.  Before finalize. */
int pgb_case_set_face_bc(pgb_case *c, int blk, int nface, int bc);
/* A face joined to a neighbour by any of the 24 orientations: orient holds
 * the reference's three digits, for each axis of blk the neighbour's axis it
 * runs along, 1-3 forward and 4-6 backward (the neighbour's face follows from
 * the digit of the face's own axis); rot, when not null, the 3 x 3 rotation
 * (row major) a rotationally periodic face turns the vectors arriving in its
 * halo by (peregrine/multiblock/interface/base.py:6-160,
 * peregrine/multiblock/collections/exchange/kernels/place.mako:3-36) */
int pgb_case_connect_oriented(pgb_case *c, int blk, int nface, int nbr, const char *orient, const double *rot);
/* register reg's halo filled from the blocks across every interface, the
 * vectors of a rotationally periodic face turned (the reference's exchange
 * of a bank, peregrine/multiblock/collections/exchange/collection.py) */
int pgb_exchange(pgb_case *c, int reg);
/* Every halo cell the case's interfaces fill, six long longs each: the
 * block and cell index (full layout) it fills, the block and cell index it
 * copies, the rotation it turns by (0 none, else 1 + its index) and 0 for
 * the first face layer, 1 for the rest; n is how many, up to cap written.
 * A host computation, before or after finalize (the reference's interior
 * exchange windows, peregrine/multiblock/collections/exchange/collection.py:63-96).
 * A partitioner lists a whole grid's entries on a case it never finalizes. */
int pgb_case_halo_entries(pgb_case *c, long long cap, long long *out, long long *n);
/* The same halo cells as the boxes the fill launches over: each face's halo
 * NG deep and each edge line one deep, as one box wherever one block holds
 * every cell's source at an index affine in the cell's.  Fourteen long longs
 * a box: the block it fills, the first cell's index there (full layout), the
 * index steps along the box's three axes (the filled block's i, j, k), the
 * extents along them, the block it copies, the first source index, the
 * source index steps along the same three axes, and the rotation (as
 * pgb_case_halo_entries').  rest is how many halo cells no box holds (the
 * fill lists those one by one).  A host computation, before or after
 * finalize; nboxes is how many there are, up to cap written.  No
 * counterpart in the reference, whose exchange copies interface windows. */
int pgb_case_halo_boxes(pgb_case *c, long long cap, long long *out, long long *nboxes, long long *rest);
/* A shard's exchange with the blocks other ranks hold: the cells it sends
 * (packs) and the halo cells it receives (unpacks), each a block and a cell
 * index, in the order the two sides agree on (the reference's message pools,
 * peregrine/multiblock/collections/exchange/pool.py:9-71).  After finalize. */
int pgb_case_set_exchange(pgb_case *c, long long nsend, const int *send_blk, const int *send_idx, long long nrecv,
                          const int *recv_blk, const int *recv_idx);
/* The register stage s of the current step reads on path, its send cells
 * packed into buf (device, ne x nsend doubles, component-major), or its
 * receive cells filled from buf (ne x nrecv); queued on the case's stream
 * (the reference's pack and place, buffer.py:7-33, place.mako). */
int pgb_exchange_pack(pgb_case *c, int stage, int path, double *buf);
int pgb_exchange_unpack(pgb_case *c, int stage, int path, const double *buf);
/* Stage s of a step on path, dt the last set (pgb_set_dt): the local halo
 * fill, the right-hand side and the combines; stages run in order, so a
 * shard exchanges its halos between them (the reference's Solver.rhs and
 * Solver.advance per stage, peregrine/integrators/rungekutta.py:33-39).
 * For cases without boundaries, double flux or sub-stepped chemistry. */
int pgb_step_stage(pgb_case *c, int s, int path);

/* the case's clock, the t boundary values read at a step's start
 * (peregrine/multiblock/solver.py:35, 355-364); a step moves it on by dt */
int pgb_set_time(pgb_case *c, double t);
int pgb_get_time(pgb_case *c, double *t);
/* the integrator's stages, in order */
int pgb_case_set_stages(pgb_case *c, const pgb_stage *stages, int nstages);
/* allocate the device arrays, build halo tables and work lists */
int pgb_case_finalize(pgb_case *c);
/* the halo depth the case uses and a block's full (halo included) extents */
int pgb_case_halo(const pgb_case *c, int *ng);
int pgb_case_device_bytes(const pgb_case *c, size_t *bytes);

/* A metric array, from the host: F order (i fastest, then j, k, components
 * outermost; numpy's order="F" of the reference's [i, j, k, comps] host view),
 * full extents with the case's halo (face arrays one plane more along their
 * axis). */
int pgb_metric_set(pgb_case *c, int blk, int which, const double *host, long count);

/* A register's interior cells, host F order (i fastest, components
 * outermost), interior only.  Logical register reg. */
int pgb_array_set(pgb_case *c, int blk, int reg, const double *host, long count);
int pgb_array_get(pgb_case *c, int blk, int reg, double *host, long count);
/* The same register with its halo: full extents (nx+4, ny+4, nz+4), F order,
 * count = ne x full cells.  The halo holds what the last right-hand side
 * left there (exchanged, or set by a boundary); its edges and corners are
 * never read (the reference's full host view, peregrine/backend/allocation.py) */
int pgb_array_get_full(pgb_case *c, int blk, int reg, double *host, long count);

/* One field of a block's eos state, full extents (nx+4, ny+4, nz+4), F order,
 * count = full cells: the state the last right-hand side or pgb_set_prims
 * formed.  Fields: 0 p, 1 T, 2 1/rho, 3 rho, 4 e, 5 cp, 6 gamma, 7 c, 8 the
 * real gas's Z, 9.. the double flux's plane (theta, eps, kappa, zeta per
 * carried species).  PGB_ERR_STATE after a batched step, which keeps no
 * state array (the reference's block state, read by its export,
 * peregrine/simulator/euler/simulator.py:66-90) */
int pgb_eos_get(pgb_case *c, int blk, int field, double *host, long count);

/* Every block's interior cells of register reg at once: the blocks' F-order
 * interior arrays end to end, in block order (count = ne x total cells). */
int pgb_state_set(pgb_case *c, int reg, const double *host, long count);
int pgb_state_get(pgb_case *c, int reg, double *host, long count);
/* page-lock a host buffer for fast copies (cudaHostRegister), and release it */
int pgb_host_register(void *host, size_t bytes);
int pgb_host_unregister(void *host);

/* Q of register reg from primitives p, u, v, w, T, Y... on the interior
 * (the reference's fromprims, peregrine/simulator/euler/kernels/state/fromprims.mako) */
int pgb_set_prims(pgb_case *c, int blk, int reg, const double *host, long count);

/* The right-hand side dQ of logical register q into logical register dq, on
 * the per-block path (halo exchange included).  Returns when queued. */
int pgb_rhs(pgb_case *c, int q, int dq);
/* The same right-hand side on a chosen path (the reference's Solver.rhs,
 * peregrine/multiblock/solver.py:270-273): PGB_PATH_PER_BLOCK as pgb_rhs,
 * PGB_PATH_PACKED the same kernels one launch a pass, PGB_PATH_BATCHED the
 * fused stage kernel itself with one combine dQ = 1 x dt x dQ at dt = 1 (the
 * halo fill of q, then one launch; PGB_ERR_UNSUPPORTED for a case the fused
 * kernel does not take).  The batched form keeps no eos state array.
 * Returns when queued. */
int pgb_rhs_path(pgb_case *c, int q, int dq, int path);
/* stage n's combines on the registers as they are, dt the last set or
 * stepped (the reference's Solver.advance, peregrine/multiblock/solver.py:276-280) */
int pgb_advance(pgb_case *c, int n);

/* nsteps steps of dt on the chosen path; graph 1 captures one step into a CUDA
 * graph and replays it.  Returns when queued on the case's stream. */
int pgb_step(pgb_case *c, double dt, int nsteps, int path, int graph);

/* nsteps steps under the cfl controller (peregrine/integrators/controllers.py:21-30,
 * peregrine/multiblock/solver.py:366-370): each step's size is
 * min(cfl / the combined CFL number per unit step of its start, dtmax), worked
 * out on the device, so the steps queue (and a graph replays them) without a
 * host round trip; the clock moves on by each step's size (pgb_get_time,
 * pgb_last_dt read them back).  Returns when queued. */
int pgb_step_cfl(pgb_case *c, double cfl, double dtmax, int nsteps, int path, int graph);
/* the largest acoustic, convective and combined CFL number per unit step over
 * every block's interior of logical register reg, out[3] (the reference's
 * cflmax, peregrine/simulator/euler/kernels/cflmax.mako, solver.py:292-296) */
int pgb_cflmax(pgb_case *c, int reg, double *out);
/* the step size of the last step queued */
int pgb_last_dt(pgb_case *c, double *dt);
/* the step scalar a right-hand side outside a step reads, the step the
 * sub-stepped chemistry integrates over (the reference's solver.dt,
 * peregrine/multiblock/solver.py:34); 0 until a step or this sets it */
int pgb_set_dt(pgb_case *c, double dt);

/* nsteps steps without a graph, a CUDA event between every launch; waits for
 * them and returns each launch's device time (ms) and kind (0 halo fill,
 * 1 fused stage or the fused passes' tile kernel, 2 per-block kernel, 3
 * combine or clock, 4 boundary pass, 5 CFL reduction, 6 sub-stepped
 * chemistry's bulk pass, 7 its stiff pass, 8 the fused passes' cell pass) in
 * launch order, up to cap launches; n is the number of launches. */
int pgb_step_timed(pgb_case *c, double dt, int nsteps, int path, float *ms, int *kind, int cap, int *n);

/* the stream the case queues on (a cudaStream_t) */
int pgb_case_stream(const pgb_case *c, void **stream);

/* the device time of the last pgb_step, milliseconds (CUDA events) */
int pgb_last_step_ms(const pgb_case *c, float *ms);

/* kernel launches the last pgb_step queued, per step */
int pgb_launches_per_step(const pgb_case *c, int path, int *count);

/* the tile shape the batched kernel uses for blk (set by the autotuner or the
 * caller); tw = th = 0 goes back to the kernel's default.  A tile the case's
 * kernel cannot take is replaced by the default when the work list is built. */
int pgb_set_tile(pgb_case *c, int blk, int tw, int th, int kchunk);
int pgb_get_tile(const pgb_case *c, int blk, int *tw, int *th, int *kchunk);

/* the uniform-metric fused kernel's instance: threads per CTA, the CTAs per
 * SM its registers are bounded for, and the widest tile its shared-memory
 * layout holds; pgb_fused_shapes lists the instances the library has, four
 * ints each (threads, minblocks, width, height) */
int pgb_set_fused_shape(pgb_case *c, int threads, int minblocks, int width);
int pgb_fused_shapes(int *shapes, int cap, int *n);
/* Whether a uniform-metric stage reads the cells past its blocks' faces
 * straight from the neighbouring blocks in place of a halo fill before it
 * (on by default).  It does so only where every face of every block is joined
 * to a neighbour low face to high face in the identity orientation, without
 * rotation, both blocks at least two cells thick across it, no exchange with
 * another case fills a halo, and the 256- or 128-thread instances run; the
 * result is the same either way.  pgb_case_halo_pull reports whether stages
 * of the finalized case read that way; before finalize, with no device
 * work, whether the wish and the blocks' faces allow it.  Other readers of a halo still get it
 * from pgb_exchange (the reference's exchange before a right-hand side,
 * peregrine/multiblock/collections/exchange/collection.py). */
int pgb_case_set_halo_pull(pgb_case *c, int on);
int pgb_case_halo_pull(const pgb_case *c, int *on);

/* The batched path's form for the case: 1 the fused stage kernel (the
 * calorically perfect single-species gas with kepaec on the cells as they
 * are), 2 the fused passes (any other ideal gas, flux function and
 * reconstruction, inviscid or viscous, with or without the coupled
 * chemistry: a cell pass and one tile kernel of every face, the divergence
 * and the combines a stage), 0 neither (boundaries, the real gas, the double
 * flux, the sub-stepped chemistry run the per-block kernels, packed).  No
 * counterpart in the reference, whose every case runs its per-kernel launches
 * (peregrine/simulator/advecdiff/simulator.py:110-124). */
int pgb_case_batched_form(const pgb_case *c, int *form);

/* whether blk runs in the uniform-metric form (1) or reads its metric arrays (0) */
int pgb_block_uniform(const pgb_case *c, int blk, int *uniform);

/* The right-hand side of one block without allocating device memory.  No
 * counterpart in the reference, which always allocates its arrays through
 * its backend.  For callers that may not call cudaMalloc or any allocating
 * library routine (torch's allocator included): code living in another
 * framework's memory pool or a fixed arena, or a host application that owns
 * all device memory.  The caller passes Q, met and dQ as device arrays, all
 * F order with the case layout's halo of two cells (full extents nx+4, ny+4,
 * nz+4, i fastest, components outermost):
 *   Q    ne = 4 + ns components, its halo filled by the caller (two layers on
 *        every face, the first layer of every edge);
 *   met  31 components: xcc (3), detJinv (1), Jinv (9, row-major), iS, jS,
 *        kS (3 each), ixc, jxc, kxc (3 each); a face of axis a is stored at
 *        the index of the cell on its high side;
 *   dQ   ne components; the interior is written, the halo left alone.
 * tables, a HOST array read during the call: Rsp, cp0, h298R, MWinv, hpoly0,
 * h298, mu0, kappa0, MWqinv, lewis (ns each), then wilkepair (ns x ns,
 * row-major).  The simulator is euler or navier-stokes, the gas calorically
 * perfect with one to three species, the flux kepaec.  The work goes on
 * stream (a cudaStream_t; NULL for the default stream) and is queued when the
 * call returns.  The scratch is one static device array of 16 MiB that every
 * GPU loading the library holds until exit; a block larger than
 * pgb_rhs_block_noalloc_max_cells(ns) cells (halo included; 52,428 for one
 * species, room for 32^3 interior cells) is refused with PGB_ERR_ARG.  The
 * first call on a device looks up the array's device address, so make it
 * before any stream capture.  Every call uses the same array and the same
 * species constants: calls that overlap on the GPU race on both, so keep
 * them ordered on one stream. */
int pgb_rhs_block_noalloc(const pgb_physics *phys, const double *tables, int nx, int ny, int nz, const double *Q,
                          const double *met, double *dQ, void *stream);
long long pgb_rhs_block_noalloc_max_cells(int ns);

/* The device's FP64 fused multiply-add rate, TFLOP/s (two flops a DFMA),
 * measured by independent FMA chains filling every SM: the denominator of the
 * FP64 roofline.  No counterpart in the reference. */
int pgb_fp64_fma_rate(double *tflops);

/* ---- serving pool ----
 * No counterpart in the reference, which runs one case per solver.  A pool
 * holds independent cases, each one block periodic onto itself, in one
 * device arena; cases are admitted while others run, and every running case
 * advances in the same launches (one launch per pass over all running
 * blocks) at one shared dt.  A block reads only its own cells, so each case's
 * result is the same as it would be alone.  The pool copies its physics,
 * tables, mechanism and RK stages from a finalized prototype case. */
typedef struct pgb_pool pgb_pool;
/* an arena of max_cells cells (halos included) and max_blocks slots (<= 65535) */
int pgb_pool_create(const pgb_case *proto, long long max_cells, int max_blocks, pgb_pool **out);
int pgb_pool_destroy(pgb_pool *p);
/* a slot for an ni x nj x nk block; PGB_ERR_NOMEM when no slot or arena
 * range is free (queue the case and admit it once another is released) */
int pgb_pool_admit(pgb_pool *p, int ni, int nj, int nk, int *slot);
/* A slot for a closed constant-volume reactor (the reference's auto-ignition
 * box, examples/autoIgnition.py:33-56): a uniform closed box has no flux
 * divergence, so the pool keeps it as one cell with no grid and steps it by
 * its eos, its finite-rate source and the stage's combines alone; its
 * primitives and register are ne values (pgb_pool_set_prims, pgb_pool_get).
 * For the coupled chemistry on the thermally perfect gas. */
int pgb_pool_admit_reactor(pgb_pool *p, int *slot);
/* the slot's metrics and primitives, laid out as pgb_metric_set's and pgb_set_prims' */
int pgb_pool_metric_set(pgb_pool *p, int slot, int which, const double *host, long count);
int pgb_pool_set_prims(pgb_pool *p, int slot, const double *host, long count);
/* the slot runs from the next step on, for nsteps RK steps */
int pgb_pool_start(pgb_pool *p, int slot, int nsteps);
/* nsteps RK steps of every running case; returns when they are done */
int pgb_pool_step(pgb_pool *p, double dt, int nsteps);
/* the slots whose steps are done (up to cap; n is how many there are) */
int pgb_pool_done(const pgb_pool *p, int *slots, int cap, int *n);
/* a slot's register over its interior, laid out as pgb_array_get's */
int pgb_pool_get(pgb_pool *p, int slot, int reg, double *host, long count);
int pgb_pool_release(pgb_pool *p, int slot);
/* the largest free arena range (cells) and the running and done counts */
int pgb_pool_info(const pgb_pool *p, long long *largest_free, int *running, int *done);
/* the last pgb_pool_step's device time (CUDA events on the pool's stream) and launches */
int pgb_pool_last(const pgb_pool *p, float *ms, int *launches);

#ifdef __cplusplus
}
#endif
#endif
