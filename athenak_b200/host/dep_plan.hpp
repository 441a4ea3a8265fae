// dep_plan.hpp -- the general deposit remap of a 3-D mesh with refinement levels, built on the
// host (the static part of AthenaK's DepRemapPlan, src/bvals/bvals_dep_general.cpp).
//
// A particle near a block face deposits into ghost cells of its own block; each ghost cell
// belongs to the active cells of the blocks it overlaps.  Every ghost cell is given to them by
// overlap volume, measured in integer cell units of the finest level (a cell of level L is
// 2^(max_level - L) units wide), so the remap conserves the deposit exactly at any level
// difference: target += (overlap volume / target cell volume) * source.  Beyond a physical x3
// face a ghost cell is mirrored back into the domain (fold) or dropped.
//
// The plan lists, per target cell, its source ghost cells and weights, targets ascending and
// each target's sources ordered by (source gid, source cell), so that the sums do not depend on
// the order in which the pairs were found.  The device applies it with dustb_ghost_add_plan
// (include/dustb.h).
#ifndef ATHENAK_B200_HOST_DEP_PLAN_HPP_
#define ATHENAK_B200_HOST_DEP_PLAN_HPP_

#include <vector>

namespace dustb_host {

struct DepPlanGeometry {
  int nx[3];          // active cells per block
  int ng;             // ghost cells
  int nmbroot[3];     // root blocks per direction
  int root_level, max_level;
  int x3mode;         // 0 periodic x3, 1 fold at physical x3 faces, 2 drop
};

struct DepPlanHost {
  std::vector<int> seg_tgt, seg_ptr, ent_src;
  std::vector<double> ent_w;
  int nbad = 0;       // source ghost cells not covered exactly once
};

// blocks: level, lx1, lx2, lx3 per block (gid order); nghbr56: 56 neighbour gids per block
// (NeighborIndex slots, -1 for none).  Returns false on invalid geometry.
bool BuildDepPlan(const DepPlanGeometry &g, int nmb, const int *lloc, const int *nghbr56,
                  DepPlanHost &out);

}  // namespace dustb_host

extern "C" {
// C entry point of BuildDepPlan for front ends without C++.  geo: nx1, nx2, nx3, ng,
// nmb_root1..3, root_level, max_level, x3mode.  counts receives nseg, nent, nbad.  With null
// outputs (or capacities below the counts) only the counts are written; returns 0, -1 for
// invalid arguments, -3 when the capacities are too small.
int dustb_host_dep_plan(const int *geo, int nmb, const int *lloc, const int *nghbr56,
                        int *counts, int *seg_tgt, int *seg_ptr, int *ent_src, double *ent_w,
                        long long cap_seg, long long cap_ent);
}

#endif  // ATHENAK_B200_HOST_DEP_PLAN_HPP_
