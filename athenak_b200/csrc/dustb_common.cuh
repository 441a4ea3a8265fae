// dustb_common.cuh -- device-side layout helpers shared by the dust drag kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dustb.h"

namespace dustb {

// RegionSize field order (src/mesh/mesh.hpp:25-29)
enum { X1MIN = 0, X2MIN = 1, X3MIN = 2, X1MAX = 3, X2MAX = 4, X3MAX = 5, DX1 = 6, DX2 = 7,
       DX3 = 8 };

// index ranges of one MeshBlock's padded arrays (mb_indcs, src/mesh/mesh.cpp:320-360)
struct Ind {
  int n1, n2, n3, is, ie, js, je, ks, ke;
  int nx1, nx2, nx3, ng, nmb, three_d, multi_d;
  __host__ __device__ long long cells() const { return (long long)n1 * n2 * n3; }
  __host__ __device__ long long at(int m, int nvar, int v, int k, int j, int i) const {
    return ((((long long)m * nvar + v) * n3 + k) * n2 + j) * (long long)n1 + i;
  }
};

inline Ind make_ind(const dustb_mesh &ms) {
  Ind d;
  d.nx1 = ms.nx1; d.nx2 = ms.multi_d ? ms.nx2 : 1; d.nx3 = ms.three_d ? ms.nx3 : 1;
  d.ng = ms.ng; d.nmb = ms.nmb; d.three_d = ms.three_d; d.multi_d = ms.multi_d;
  d.n1 = ms.nx1 + 2 * ms.ng;
  d.n2 = ms.multi_d ? ms.nx2 + 2 * ms.ng : 1;
  d.n3 = ms.three_d ? ms.nx3 + 2 * ms.ng : 1;
  d.is = ms.ng; d.ie = d.is + d.nx1 - 1;
  d.js = ms.multi_d ? ms.ng : 0; d.je = d.js + d.nx2 - 1;
  d.ks = ms.three_d ? ms.ng : 0; d.ke = d.ks + d.nx3 - 1;
  return d;
}

// PMWeights (src/dust/dust.hpp:1088-1111), FP64, operation for operation.
__device__ __forceinline__ void pm_weights(double x, double xmin, double xmax, int nx, int is,
                                           int scheme, int &ip, double w[3]) {
  double cell = (x - xmin) * ((double)nx / (xmax - xmin));
  int ig = (int)(cell + 1.0) - 1;
  double del = cell - ((double)ig + 0.5);
  ip = ig + is;
  if (scheme == 0) {
    w[0] = 0.0; w[1] = 1.0; w[2] = 0.0;
  } else if (scheme == 1) {
    w[0] = fmax(0.0, -del); w[1] = 1.0 - fabs(del); w[2] = fmax(0.0, del);
  } else {
    w[0] = 0.5 * ((0.5 - del) * (0.5 - del));
    w[1] = 0.75 - del * del;
    w[2] = 0.5 * ((0.5 + del) * (0.5 + del));
  }
}

__device__ __forceinline__ void report(unsigned int *err, unsigned int bit) {
  if (err) atomicOr(err, bit);
}

// the 26 same-level directions in NeighborIndex(ox1,ox2,ox3,0,0) order
// (src/mesh/nghbr_index.hpp:29-55): the order RecvAndSumDeposit sums its buffers in
__constant__ const signed char kDirOrder[26][3] = {
  {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0},
  {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0},
  {0, 0, -1}, {0, 0, 1},
  {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {1, 0, 1},
  {0, -1, -1}, {0, 1, -1}, {0, -1, 1}, {0, 1, 1},
  {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
  {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};

__host__ __device__ inline int dir_slot(int o1, int o2, int o3) {
  return (o3 + 1) * 9 + (o2 + 1) * 3 + (o1 + 1);
}

// the slot of direction (ix, iy, iz) and sub-slot (n1, n2) among the 56 neighbours of a block of
// a refined 3-D mesh (NeighborIndex, src/mesh/nghbr_index.hpp:29-60): x1 faces 0-7, x2 faces
// 8-15, x1x2 edges 16-23, x3 faces 24-31, x3x1 edges 32-39, x2x3 edges 40-47, corners 48-55
__host__ __device__ inline int nbr_slot(int ix, int iy, int iz, int n1, int n2) {
  const int ax = ix < 0 ? -ix : ix, ay = iy < 0 ? -iy : iy;
  if (iz == 0) {
    if (ix * iy == 0) return ax * 2 * (ix + 1) + ay * 2 * (iy + 5) + n1 + 2 * n2;
    return 16 + (ix + 1) + 2 * (iy + 1) + n1;
  }
  if (ix * iy == 0) return 24 + ax * (ix + 9) + ay * (iy + 17) + 2 * (iz + 1) + n1 + 2 * n2;
  return 48 + (ix + 1) / 2 + (iy + 1) + 2 * (iz + 1);
}


// SetNewPrtclGID's neighbour slot on a refined mesh (src/bvals/bvals_part.cpp:312-394): the slot
// of the crossing direction (ix, iy, iz); a finer neighbour's sub-slot from the half (fx, fy,
// fz) of the block the particle leaves from; the first filled sub-slot of the direction; an
// empty edge or corner is covered by a coarser block stored under the lower-dimensional
// direction that keeps the components leaving this block's parent.  nb: the block's 56 slot
// gids, lev: block levels (by gid - gids), mb: the block's RegionSize, x?min: the mesh's
// lower corner.  -1 if no slot holds a block.
__device__ inline int ml_route_slot(const int *nb, const int *lev, int gids, int mylevel,
                                    const double *mb, double x1min, double x2min, double x3min,
                                    int ix, int iy, int iz, int fx, int fy, int fz) {
  auto lev_of = [&](int slot) {
    const int g = nb[slot] - gids;
    return (nb[slot] >= 0 && g >= 0) ? lev[g] : -1;
  };
  auto filled = [&](int jx, int jy, int jz, int k) {
    const int nd = abs(jx) + abs(jy) + abs(jz);
    const int end = nbr_slot(jx, jy, jz, 0, 0) + ((nd == 1) ? 4 : ((nd == 2) ? 2 : 1));
    for (; k < end; ++k)
      if (nb[k] >= 0) return k;
    return -1;
  };
  auto coarse_cover = [&](int jx, int jy, int jz) {
    const double lx = mb[X1MAX] - mb[X1MIN], ly = mb[X2MAX] - mb[X2MIN], lz = mb[X3MAX] - mb[X3MIN];
    const int l1 = (int)floor((mb[X1MIN] - x1min) / lx + 0.5);
    const int l2 = (int)floor((mb[X2MIN] - x2min) / ly + 0.5);
    const int l3 = (int)floor((mb[X3MIN] - x3min) / lz + 0.5);
    const int kx = (jx == 0 || ((l1 & 1) == ((jx > 0) ? 1 : 0))) ? jx : 0;
    const int ky = (jy == 0 || ((l2 & 1) == ((jy > 0) ? 1 : 0))) ? jy : 0;
    const int kz = (jz == 0 || ((l3 & 1) == ((jz > 0) ? 1 : 0))) ? jz : 0;
    if (abs(kx) + abs(ky) + abs(kz) == 0 || (kx == jx && ky == jy && kz == jz)) return -1;
    return filled(kx, ky, kz, nbr_slot(kx, ky, kz, 0, 0));
  };
  int s;
  if (iz == 0) {
    if (iy == 0) {                                          // x1 face
      s = nbr_slot(ix, 0, 0, 0, 0);
      if (lev_of(s) > mylevel) s = nbr_slot(ix, 0, 0, fy, fz);
      s = filled(ix, 0, 0, s);
    } else if (ix == 0) {                                   // x2 face
      s = nbr_slot(0, iy, 0, 0, 0);
      if (lev_of(s) > mylevel) s = nbr_slot(0, iy, 0, fx, fz);
      s = filled(0, iy, 0, s);
    } else {                                                // x1x2 edge
      s = nbr_slot(ix, iy, 0, 0, 0);
      if (lev_of(s) > mylevel) s = nbr_slot(ix, iy, 0, fz, 0);
      s = filled(ix, iy, 0, s);
      if (s < 0) s = coarse_cover(ix, iy, 0);
    }
  } else if (iy == 0) {
    if (ix == 0) {                                          // x3 face
      s = nbr_slot(0, 0, iz, 0, 0);
      if (lev_of(s) > mylevel) s = nbr_slot(0, 0, iz, fx, fy);
      s = filled(0, 0, iz, s);
    } else {                                                // x3x1 edge
      s = nbr_slot(ix, 0, iz, 0, 0);
      if (lev_of(s) > mylevel) s = nbr_slot(ix, 0, iz, fy, 0);
      s = filled(ix, 0, iz, s);
      if (s < 0) s = coarse_cover(ix, 0, iz);
    }
  } else if (ix == 0) {                                     // x2x3 edge
    s = nbr_slot(0, iy, iz, 0, 0);
    if (lev_of(s) > mylevel) s = nbr_slot(0, iy, iz, fx, 0);
    s = filled(0, iy, iz, s);
    if (s < 0) s = coarse_cover(0, iy, iz);
  } else {                                                  // corner
    s = filled(ix, iy, iz, nbr_slot(ix, iy, iz, 0, 0));
    if (s < 0) s = coarse_cover(ix, iy, iz);
  }
  return s;
}
}  // namespace dustb

// host-side error bookkeeping shared by the translation units
namespace dustb_host {
void set_error(const char *what, cudaError_t e);
void set_message(const char *what);
int launch_status(const char *what);
}  // namespace dustb_host
