// Device layout of a case's arrays.
//
// Every register (Q, Q1, ... in the reference's naming,
// peregrine/launch/arrays.py:37-39) is one allocation holding every block.
// With cv[b] the cells of the blocks before b and C components per cell,
// block b's component c starts at C * cv[b] + c * vol[b] doubles, and its cell
// (i, j, k), counted from the first halo layer, sits at i + X * (j + Y * k)
// inside that.  i runs fastest, components outermost: the reference's device
// F order (peregrine/backend/device/backend.py:57-58), with the blocks laid
// end to end.  The metric arrays share the layout, 31 components per cell.
// A face array of axis a keeps face f at the index of the cell on its high
// side (the reference indexes a face like the cell to its right,
// peregrine/launch/policy.py:78-86), so faces use the cell layout too.
#pragma once
#include <cstdint>

namespace pgb {

constexpr int NG = 2;  // halo layers: the fused stage's stencil reaches two cells

// metric components inside the metric allocation
enum {
  M_XCC = 0, M_DETJINV = 3, M_JINV = 4, M_S = 13, M_XF = 22, M_NCOMP = 31
};

struct BlockDev {
  int nx, ny, nz;     // interior cells
  int X, Y, Z;        // full extents, nx + 2 NG ...
  long long vol;      // X * Y * Z
  long long cv;       // cells of the blocks before this one
  int uniform;        // 1: the metrics are the per-axis constants below
  // uniform form, every value read off the block's own metric arrays
  double S[3];        // the area vector's normal component of an a-face
  double detJinv;
  double Jd[3];       // inverse Jacobian diagonal
  double ex[3];       // xcc(R) - xcc(L) along a
  double xL[3];       // xf - xcc(L) along a
  double xR[3];       // xf - xcc(R) along a
  // per-axis face geometry alpha damping forms, precomputed from the above
  double damp[3];     // alpha / |e . n| for an a-face (the normal is the axis)
};

__host__ __device__ __forceinline__ long long cell_index(const BlockDev &b, int fi, int fj, int fk) {
  return (long long)fi + (long long)b.X * ((long long)fj + (long long)b.Y * fk);
}

// The per-cell state of the per-block path, fields of one cell SW apart in
// vol-strided planes: the EosState (p, T, rhoinv, rho, e, cp, gamma, c), the
// real gas's root Z, and the double flux's tangent plane of rho e
// (theta, eps, kappa, zeta[ns - 1]) (peregrine/simulator/mixture/eos/base.py:85-86,
// realgas/model.py:31-34, realgasdf/model.py:8-10)
constexpr int SW = 24;
enum { ST_Z = 8, ST_THETA = 9, ST_EPS = 10, ST_KAPPA = 11, ST_ZETA = 12 };

// Where a per-block kernel's thread works: its block and its index t in the
// pass's range over that block.  With a tile table (a packed launch over many
// blocks), CTA x does tile ctab[x].y of block row ctab[x].x, so a launch has
// exactly the CTAs its blocks need; without one, the block is b plus the grid
// row and the tile the CTA's x.  The kernel names its block index b, its
// descriptor table blks and its tile table ctab.
#define PGB_WHERE(B, t)                                                                              \
  const int2 where_ = ctab ? ctab[blockIdx.x] : make_int2(b + (int)blockIdx.y, (int)blockIdx.x); \
  const BlockDev &B = blks[where_.x];                                                                \
  const long long t = (long long)where_.y * blockDim.x + threadIdx.x

// one cell of a halo filled from another cell: each side's block start in
// cells (cv), its cell index inside the block and its component stride
// (vol); rot, when not 0, the rotation (rot - 1 in the case's table) a
// rotationally periodic interface turns the cell's vectors by
struct HaloEntry {
  long long dcv, scv;
  int didx, sidx, dvol, svol;
  int rot;
};

// A box of halo cells of one block whose sources all lie in one block, the
// source index an affine map of the destination cell: a face's halo NG deep,
// an edge line one deep.  The box runs i fastest in the destination, so a
// warp's threads write neighbouring cells; t = x0 + n0 (x1 + n1 x2) is the
// thread's cell in it, the indices d0 + x . dst and s0 + x . sst.
struct HaloPatch {
  long long dcv, scv;
  int dvol, svol;
  int d0, s0;
  int dst[3], sst[3];
  int n0, n1, cells;
  int rot;
};

// what k_halo turns with an entry's rotation: nothing, the vector at a
// component (Q's momentum at 1), or the gradients' tensor (each row's three
// directions, and the velocity rows u, v, w down every direction)
enum { HALO_SCALARS = -1, HALO_TENSOR = -2 };

// a fused work item: a column of tw x th cells of one block over k0 .. k1 - 1
struct TileDev {
  int blk;
  short i0, j0, tw, th, k0, k1;
};

}  // namespace pgb
