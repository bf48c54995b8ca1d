// Fusion planner: groups a lowered gate list into stages.
//
// A stage owns a set S of m index bits (always including the L lowest bits,
// so that every tile is made of contiguous runs of 2^L amplitudes).  The
// state is streamed through shared memory one tile at a time -- a tile is
// the 2^m amplitudes that agree on every bit outside S -- and all gates of
// the stage, whose bits lie in S, are applied to the tile before it is
// written back: one HBM read and write of the state per stage instead of
// one per gate.
//
// Gates are taken greedily in circuit order.  A gate joins the current
// stage if its bits are in S or can still be added to S (|S| <= m) and none
// of its bits is "blocked"; a gate that cannot join blocks its bits, so no
// later gate that shares a bit with it moves ahead of it.  Gates acting on
// disjoint bits commute, so the stage order is a valid reordering of the
// circuit.
#pragma once

#include <cstdint>
#include <vector>
#include "lower.hpp"

namespace qsv {

struct Stage {
  int m = 0;                  // tile bits
  int bits[64];               // local bit j -> global bit (ascending)
  std::vector<int> gates;     // indices into the lowered list, in order
};

inline uint64_t gate_bits(const Lowered& L) {
  switch (L.shape) {
    case SH_PAIR:
    case SH_HALF:
      return 1ull << L.t0;
    case SH_QUAD:
    case SH_CPAIR:
    case SH_CHALF:
    case SH_SWAP:
      return (1ull << L.t0) | (1ull << L.t1);
    case SH_RED:
      return L.gen.f | L.gen.zy | L.gen.pm;
    default:
      return 0;
  }
}

// Upper bound of the device plan bytes one item adds to its stage: its op
// (24 B), a pass descriptor (80 B, as if the op had a pass to itself) and
// its coefficients of elem_bytes each.
inline size_t plan_bytes_of(const Lowered& L, size_t elem_bytes) {
  int nc = 0;
  switch (L.shape) {
    case SH_PAIR: case SH_CPAIR: nc = 4; break;
    case SH_QUAD: nc = 16; break;
    case SH_HALF: case SH_CHALF: case SH_SWAP: nc = 1; break;
    case SH_RED: nc = 2; break;
    default: break;
  }
  return 24 + 80 + size_t(nc) * elem_bytes;
}

// Builds stages for an n-qubit state with tiles of 2^m amplitudes whose
// lowest `low` bits are contiguous.  max_gates bounds the gates of a stage,
// max_red its gradient reductions (SH_RED items) and max_bytes the plan
// bytes of its items (plan_bytes_of with elem_bytes); 0 = unbounded.
std::vector<Stage> plan_stages(const std::vector<Lowered>& gates, int n, int m,
                               int low, int max_gates, int max_red = 0,
                               size_t max_bytes = 0, size_t elem_bytes = 16);

// A register pass inside a stage: r tile bits (ascending local positions)
// whose 2^r amplitudes one thread holds in registers while it applies the
// pass's ops (indices into the stage's op list, in order).
struct Pass {
  int r = 0;
  int pos[8];
  std::vector<int> ops;
};

// Groups a stage's ops (given by their local bit masks, in order) into
// register passes of at most r bits, with the same blocking rule as
// plan_stages, so each pass is a valid reordering of commuting ops.  Every
// pass is padded to exactly r bits (the lowest unused local bits; m >= r).
// search = false: each pass takes ops in order while their bits fit in r
// (greedy).  search = true (passes multiplied out into dense matrices, whose
// cost does not depend on how many ops they hold): each pass's r bits are
// the set, among the greedy one and every r-bit set holding the first
// remaining op, after which the greedy planner needs the fewest passes for
// the rest of the stage (ties keep the greedy set).
std::vector<Pass> plan_passes(const std::vector<uint32_t>& op_bits, int m, int r,
                              bool search = false);

}  // namespace qsv
