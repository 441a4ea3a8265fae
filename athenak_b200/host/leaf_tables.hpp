// leaf_tables.hpp -- the block geometry of the refinable clouds' leaf traversal on a refined 3-D
// mesh, built on the host (DustGasDrag::BuildLeafTraversal3D, src/dust/dust_cloud3d.cpp:357-860,
// one rank: every block is a local slot).
//
// A cloud anchored at block m is integrated over the leaf cells of m and of the blocks next to
// it.  Per block the tables hold its box in cells of the finest level (fbox), its level above
// the root (blev), its distinct neighbours from the 56 NeighborIndex slots with the periodic
// shift that places each next to it (nb, nbs), the finest level among the block and its
// neighbours (nbmax), the ring of finest cells those neighbours certainly hold (safe: the
// narrowest neighbour width per direction, 0 when some cell of that ring is not held), and the
// sorted logical-location keys of all blocks (lockey, locblk) for the global owner search.
#ifndef ATHENAK_B200_HOST_LEAF_TABLES_HPP_
#define ATHENAK_B200_HOST_LEAF_TABLES_HPP_

#include <cstdint>
#include <vector>

namespace dustb_host {

constexpr int kLeafMaxNb = 64;   // distinct neighbours of a 3-D block (56 at most)

struct LeafGeometry {
  int nx[3];          // active cells per block
  int nmbroot[3];     // root blocks per direction
  int root_level, max_level;
  int x3per;          // 1: periodic x3; 0: physical x3 faces
};

struct LeafTablesHost {
  int nlev = 0;
  int nfine[3] = {0, 0, 0};
  std::vector<int> fbox, blev, nnb, nb, nbs, nbmax, safe, locblk;
  std::vector<std::int64_t> lockey;
  int nunsafe = 0;     // blocks whose neighbours do not certainly hold a ring
};

// the logical-location key (level above the root, lx1, lx2, lx3), 19 bits per index
inline std::int64_t LeafLocKey(int l, int lx1, int lx2, int lx3) {
  return ((std::int64_t)l << 57) | ((std::int64_t)lx3 << 38) | ((std::int64_t)lx2 << 19) |
         (std::int64_t)lx1;
}

// lloc: level, lx1, lx2, lx3 per block (gid order); nghbr56: 56 neighbour gids per block
// (NeighborIndex slots, -1 for none).  Returns false on invalid geometry (a block finer than
// max_level, more than kLeafMaxNb distinct neighbours, a neighbour gid out of range).
bool BuildLeafTables(const LeafGeometry &g, int nmb, const int *lloc, const int *nghbr56,
                     LeafTablesHost &out);

}  // namespace dustb_host

extern "C" {
// C entry point of BuildLeafTables.  geo: nx1..3, nmb_root1..3, root_level, max_level, x3per.
// info receives nlev, nfine1..3, nunsafe.  The outputs are sized by the caller: fbox nmb x 6,
// blev, nnb, nbmax, locblk nmb, nb nmb x 64, nbs nmb x 64 x 3, safe nmb x 3, lockey nmb.  Returns
// 0, or -1 for invalid arguments or geometry.
int dustb_host_leaf_tables(const int *geo, int nmb, const int *lloc, const int *nghbr56,
                           int *info, int *fbox, int *blev, int *nnb, int *nb, int *nbs,
                           int *nbmax, int *safe, long long *lockey, int *locblk);
}

#endif  // ATHENAK_B200_HOST_LEAF_TABLES_HPP_
