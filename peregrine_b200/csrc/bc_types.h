// The boundary tables as the device reads them: the value programs, the
// entries (a kind and where each of its values' programs starts) and the
// block faces a boundary pass covers.  Plain structs the host fills, shared by
// the library's translation units.
#pragma once
#include "pgb200.h"
#include "physics.cuh"

namespace pgb {

// the most values an entry gives: p u v w T and the carried species
constexpr int BC_MAXV = 5 + MAXNS - 1;

struct BcOp {
  int op;      // PGB_OP_*
  int pad;
  double arg;  // CONST's operand
};

// one bcvals entry: its kind and its values, value v the program
// ops[start[v] .. start[v + 1])
struct BcEntry {
  int kind;
  int nval;
  int start[BC_MAXV + 1];
};

// one block face of a boundary pass.  A pass's table lists its faces in the
// order of their threads and ends with a sentinel whose start is the pass's
// thread count.
struct BcFace {
  int blk;
  int face;   // 0..5: i-low, i-high, j-low, j-high, k-low, k-high
  int entry;
  int pad;
  long long start;  // the face's first thread in the pass
};

inline __host__ __device__ bool bc_is_wall(int kind) {
  return kind >= PGB_BC_SLIP_ADIA_WALL && kind <= PGB_BC_MOV_ISOT_WALL;
}

// the values a kind reads before the species, and whether the carried
// species' mass fractions follow (the inlets; peregrine/simulator/euler/bcs.py:5-8)
inline int bc_head_values(int kind) {
  switch (kind) {
    case PGB_BC_SLIP_ISOT_WALL:
    case PGB_BC_NOSLIP_ISOT_WALL:
    case PGB_BC_SUB_OUT_FP: return 1;
    case PGB_BC_MOV_ADIA_WALL: return 3;
    case PGB_BC_MOV_ISOT_WALL:
    case PGB_BC_SUB_IN_FVT: return 4;
    case PGB_BC_SUP_IN_FA: return 5;
    case PGB_BC_SUB_IN_FTPTT:
    case PGB_BC_SUB_IN_FMT: return 2;
    default: return 0;
  }
}

inline bool bc_is_inlet(int kind) { return kind >= PGB_BC_SUB_IN_FVT && kind <= PGB_BC_SUB_IN_FMT; }

}  // namespace pgb
