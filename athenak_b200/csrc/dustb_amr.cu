// dustb_amr.cu -- the copy exchange of a cell-centred field on a refined 3-D mesh (blocks of
// several levels): the ghost cells of u* (and of any field the drag gathers from) filled from
// neighbours of the same, a coarser or a finer level.
//
// The steps are those of AthenaK's multilevel cell-centred boundary values, which the dust
// module's u* exchange uses (DustGasDrag::SendUstar / RecvUstar / FinishUstarGhosts,
// src/dust/dust_tasks.cpp:262-442):
//   1. restriction of every block's active cells into its coarse array (the mean of the 8
//      fine cells; MeshRefinement::RestrictCC, src/mesh/mesh_refinement.cpp:1829-1880);
//   2. the exchange proper (MeshBoundaryValuesCC::PackAndSendCC / RecvAndUnpackCC,
//      src/bvals/bvals_cc.cpp:53-460): a same-level neighbour's active strip into the ghost
//      cells, a finer neighbour's coarse array (its restriction) into the ghost cells, a
//      coarser neighbour's active cells into the coarse array's ghost cells -- with the index
//      boxes of MeshBoundaryValuesCC::InitSendIndices / InitRecvIndices
//      (src/bvals/buffs_cc.cpp:28-410), the box of each of the 56 neighbour slots;
//   3. the coarse array's ghost cells next to same-level neighbours from the fine ghost cells
//      just received (FillCoarseInBndryCC, src/bvals/prolongation.cpp:29-120);
//   4. prolongation of the coarse ghost cells next to coarser neighbours into the fine ghost
//      cells with min-mod limited slopes (ProlongateCC / ProlongCC,
//      src/bvals/prolongation.cpp:145-230, src/mesh/prolongation.hpp:21-80).
// On one device the exchange is a pull: every receiving (block, slot) copies from the box of
// its neighbour's slot that points back to it (the neighbour's dest slot, the rules of
// MeshBlock::SetNeighbors, src/mesh/meshblock.cpp:142-420).  The coarse arrays are scratch
// of the caller, cleared at every call.
#include <cuda_runtime.h>

#include "dustb_common.cuh"

using namespace dustb;

namespace {

constexpr int kThr = 256;

inline unsigned grid_for(long long n) {
  long long b = (n + kThr - 1) / kThr;
  return (unsigned)(b < 1 ? 1 : b);
}

// (ox1, ox2, ox3, f1, f2) of the 56 neighbour slots, in the loops of
// MeshBoundaryValues::InitializeBuffers (src/bvals/bvals.cpp:323-420)
struct SlotTab { signed char o[56][5]; };

SlotTab make_slots() {
  SlotTab t{};
  auto put = [&](int ix, int iy, int iz, int a, int b) {
    const int s = nbr_slot(ix, iy, iz, a, b);
    t.o[s][0] = (signed char)ix; t.o[s][1] = (signed char)iy; t.o[s][2] = (signed char)iz;
    t.o[s][3] = (signed char)a; t.o[s][4] = (signed char)b;
  };
  for (int n = -1; n <= 1; n += 2)
    for (int fz = 0; fz < 2; ++fz) for (int fy = 0; fy < 2; ++fy) put(n, 0, 0, fy, fz);
  for (int m = -1; m <= 1; m += 2)
    for (int fz = 0; fz < 2; ++fz) for (int fx = 0; fx < 2; ++fx) put(0, m, 0, fx, fz);
  for (int m = -1; m <= 1; m += 2)
    for (int n = -1; n <= 1; n += 2) for (int fz = 0; fz < 2; ++fz) put(n, m, 0, fz, 0);
  for (int l = -1; l <= 1; l += 2)
    for (int fy = 0; fy < 2; ++fy) for (int fx = 0; fx < 2; ++fx) put(0, 0, l, fx, fy);
  for (int l = -1; l <= 1; l += 2)
    for (int n = -1; n <= 1; n += 2) for (int fy = 0; fy < 2; ++fy) put(n, 0, l, fy, 0);
  for (int l = -1; l <= 1; l += 2)
    for (int m = -1; m <= 1; m += 2) for (int fx = 0; fx < 2; ++fx) put(0, m, l, fx, 0);
  for (int l = -1; l <= 1; l += 2)
    for (int m = -1; m <= 1; m += 2) for (int n = -1; n <= 1; n += 2) put(n, m, l, 0, 0);
  return t;
}

// the index ranges of one block: fine (is..ie per direction), coarse (cis..cie), the coarse
// array's extents, the ghost width
struct Geo3 {
  int nx[3], cnx[3], ng, is[3], ie[3], cis[3], cie[3];
  int n[3], cn[3];                        // fine and coarse array extents
  long long fcells, ccells;
};

Geo3 make_geo3(const dustb_mesh &ms) {
  Geo3 g;
  const int nx[3] = {ms.nx1, ms.nx2, ms.nx3};
  g.ng = ms.ng;
  for (int d = 0; d < 3; ++d) {
    g.nx[d] = nx[d]; g.cnx[d] = nx[d] / 2;
    g.is[d] = ms.ng; g.ie[d] = ms.ng + nx[d] - 1;
    g.cis[d] = ms.ng; g.cie[d] = ms.ng + g.cnx[d] - 1;
    g.n[d] = nx[d] + 2 * ms.ng; g.cn[d] = g.cnx[d] + 2 * ms.ng;
  }
  g.fcells = (long long)g.n[0] * g.n[1] * g.n[2];
  g.ccells = (long long)g.cn[0] * g.cn[1] * g.cn[2];
  return g;
}

struct Box { int lo[3], hi[3]; };

// which sub-slot index selects the half of a direction left free by the slot: x1 takes f1,
// x2 f1 when x1 is crossed (else f2), x3 f1 when x1 and x2 are crossed (else f2)
__device__ __forceinline__ int free_f(const int o[3], int f1, int f2, int d) {
  if (d == 0) return f1;
  if (d == 1) return (o[0] != 0) ? f1 : f2;
  return (o[0] != 0 && o[1] != 0) ? f1 : f2;
}

// InitSendIndices (src/bvals/buffs_cc.cpp:28-150), 3-D: kind 0 same level (from the fine
// array), 1 to a coarser neighbour (from the coarse array), 2 to a finer neighbour (from the
// fine array, the internal edges of faces and corners of edges added)
__device__ Box send_box(const Geo3 &g, const int o[3], int f1, int f2, int kind) {
  Box b;
  const int ng1 = g.ng - 1;
  for (int d = 0; d < 3; ++d) {
    const int s = (kind == 1) ? g.cis[d] : g.is[d], e = (kind == 1) ? g.cie[d] : g.ie[d];
    b.lo[d] = (o[d] > 0) ? e - ng1 : s;
    b.hi[d] = (o[d] < 0) ? s + ng1 : e;
    if (kind == 2 && o[d] == 0) {
      if (free_f(o, f1, f2, d) == 1) b.lo[d] += g.cnx[d] - g.ng;
      else b.hi[d] -= g.cnx[d] - g.ng;
    }
  }
  return b;
}

// InitRecvIndices (src/bvals/buffs_cc.cpp:164-360), 3-D: kind 0 from the same level (into the
// fine ghost cells), 1 from a coarser neighbour (into the coarse array, widened by ng over the
// free halves), 2 from a finer neighbour (into the fine ghost cells of that sub-block), 3 the
// prolongation box (coarse cells, as kind 1 with ng/2)
__device__ Box recv_box(const Geo3 &g, const int o[3], int f1, int f2, int kind) {
  Box b;
  const int w = (kind == 3) ? g.ng / 2 : g.ng;
  for (int d = 0; d < 3; ++d) {
    const bool coarse = (kind == 1 || kind == 3);
    const int s = coarse ? g.cis[d] : g.is[d], e = coarse ? g.cie[d] : g.ie[d];
    if (o[d] > 0) { b.lo[d] = e + 1; b.hi[d] = e + w; continue; }
    if (o[d] < 0) { b.lo[d] = s - w; b.hi[d] = s - 1; continue; }
    b.lo[d] = s; b.hi[d] = e;
    const int f = free_f(o, f1, f2, d);
    if (kind == 1 || kind == 3) {
      if (f == 0) b.hi[d] += w; else b.lo[d] -= w;
    } else if (kind == 2) {
      if (f == 1) b.lo[d] += g.cnx[d]; else b.hi[d] -= g.cnx[d];
    }
  }
  return b;
}

// the slot of the neighbour in slot (o, f1, f2) that points back to this block
// (MeshBlock::SetNeighbors' dest): same level the opposite direction; a finer neighbour sees
// this block in the sub-slot of its own position, (f1, f2); a coarser neighbour sees it in the
// sub-slot of this block's position on the shared face or edge
__device__ int dest_slot(const int o[3], int f1, int f2, int rel, const int myf[3]) {
  const int nd = abs(o[0]) + abs(o[1]) + abs(o[2]);
  if (rel == 0 || nd == 3) return nbr_slot(-o[0], -o[1], -o[2], 0, 0);
  if (rel > 0) return nbr_slot(-o[0], -o[1], -o[2], f1, nd == 1 ? f2 : 0);
  int a = 0, b = 0;
  if (nd == 1) {
    const int t1 = (o[0] != 0) ? 1 : 0, t2 = (o[2] != 0) ? 1 : 2;
    a = myf[t1]; b = myf[t2];
  } else {
    a = myf[(o[0] == 0) ? 0 : ((o[1] == 0) ? 1 : 2)];
  }
  return nbr_slot(-o[0], -o[1], -o[2], a, b);
}

struct AmrArgs {
  SlotTab tab;
  Geo3 g;
  int nmb, nvar, gids;
  const int *nb, *lev;
  const double *mb;
  double x1min, x2min, x3min;
  double *a, *ca;
};

__device__ __forceinline__ long long fidx(const AmrArgs &A, int m, int v, int k, int j, int i) {
  return (((long long)m * A.nvar + v) * A.g.n[2] + k) * (long long)(A.g.n[1] * A.g.n[0]) +
         (long long)j * A.g.n[0] + i;
}
__device__ __forceinline__ long long cidx(const AmrArgs &A, int m, int v, int k, int j, int i) {
  return (((long long)m * A.nvar + v) * A.g.cn[2] + k) * (long long)(A.g.cn[1] * A.g.cn[0]) +
         (long long)j * A.g.cn[0] + i;
}

// the parity of a block's logical location per direction, from its box (as SetNewPrtclGID's
// coarse_cover forms the location, src/bvals/bvals_part.cpp:335-340)
__device__ __forceinline__ void parity(const AmrArgs &A, int m, int f[3]) {
  const double *s = A.mb + (long long)m * 9;
  const double lo[3] = {A.x1min, A.x2min, A.x3min};
  for (int d = 0; d < 3; ++d) {
    const double l = s[3 + d] - s[d];
    f[d] = ((int)floor((s[d] - lo[d]) / l + 0.5)) & 1;
  }
}

// the mean of the 8 fine cells under coarse cell (k, j, i), summed in the reference's order
__device__ __forceinline__ double restrict8(const AmrArgs &A, int m, int v, int k, int j, int i) {
  const int fi = (i - A.g.cis[0]) * 2 + A.g.is[0];
  const int fj = (j - A.g.cis[1]) * 2 + A.g.is[1];
  const int fk = (k - A.g.cis[2]) * 2 + A.g.is[2];
  const double *a = A.a;
  return 0.125 * (a[fidx(A, m, v, fk, fj, fi)] + a[fidx(A, m, v, fk, fj, fi + 1)] +
                  a[fidx(A, m, v, fk, fj + 1, fi)] + a[fidx(A, m, v, fk, fj + 1, fi + 1)] +
                  a[fidx(A, m, v, fk + 1, fj, fi)] + a[fidx(A, m, v, fk + 1, fj, fi + 1)] +
                  a[fidx(A, m, v, fk + 1, fj + 1, fi)] + a[fidx(A, m, v, fk + 1, fj + 1, fi + 1)]);
}

// 1. RestrictCC over every block's active coarse cells
__global__ void k_restrict(AmrArgs A) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int c0 = A.g.cnx[0], c1 = A.g.cnx[1], c2 = A.g.cnx[2];
  const long long per = (long long)c0 * c1 * c2;
  if (t >= per * A.nvar * A.nmb) return;
  long long r = t;
  const int i = (int)(r % c0) + A.g.cis[0]; r /= c0;
  const int j = (int)(r % c1) + A.g.cis[1]; r /= c1;
  const int k = (int)(r % c2) + A.g.cis[2]; r /= c2;
  const int v = (int)(r % A.nvar);
  const int m = (int)(r / A.nvar);
  A.ca[cidx(A, m, v, k, j, i)] = restrict8(A, m, v, k, j, i);
}

// 2. the exchange, pulled by every receiving (block, slot); emax elements per (block, slot,
// variable), the box's own count checked
__global__ void k_exchange(AmrArgs A, int emax) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)56 * A.nvar * emax;
  if (t >= per * A.nmb) return;
  const int m = (int)(t / per);
  long long r = t - (long long)m * per;
  const int n = (int)(r / ((long long)A.nvar * emax)); r -= (long long)n * A.nvar * emax;
  const int v = (int)(r / emax);
  const int e = (int)(r - (long long)v * emax);
  const int gs = A.nb[(long long)m * 56 + n];
  if (gs < 0) return;
  const int s = gs - A.gids;
  if (s < 0 || s >= A.nmb) return;
  const int o[3] = {A.tab.o[n][0], A.tab.o[n][1], A.tab.o[n][2]};
  const int f1 = A.tab.o[n][3], f2 = A.tab.o[n][4];
  const int rel = A.lev[s] - A.lev[m];                 // > 0: the neighbour is finer
  const int rk = (rel < 0) ? 1 : ((rel == 0) ? 0 : 2);
  const Box rb = recv_box(A.g, o, f1, f2, rk);
  const int ni = rb.hi[0] - rb.lo[0] + 1, nj = rb.hi[1] - rb.lo[1] + 1;
  const int nk = rb.hi[2] - rb.lo[2] + 1;
  if (e >= ni * nj * nk) return;
  const int di = e % ni, dj = (e / ni) % nj, dk = e / (ni * nj);
  int myf[3];
  parity(A, m, myf);
  const int ns = dest_slot(o, f1, f2, rel, myf);
  const int so[3] = {A.tab.o[ns][0], A.tab.o[ns][1], A.tab.o[ns][2]};
  // the sender's view: this block is coarser (rel > 0), the same level or finer
  const int sk = (rel > 0) ? 1 : ((rel == 0) ? 0 : 2);
  const Box sb = send_box(A.g, so, A.tab.o[ns][3], A.tab.o[ns][4], sk);
  const int si = sb.lo[0] + di, sj = sb.lo[1] + dj, sk3 = sb.lo[2] + dk;
  const double val = (sk == 1) ? A.ca[cidx(A, s, v, sk3, sj, si)] : A.a[fidx(A, s, v, sk3, sj, si)];
  const int ii = rb.lo[0] + di, jj = rb.lo[1] + dj, kk = rb.lo[2] + dk;
  if (rk == 1) A.ca[cidx(A, m, v, kk, jj, ii)] = val;
  else A.a[fidx(A, m, v, kk, jj, ii)] = val;
}

// 3. FillCoarseInBndryCC: the coarse ghost cells next to same-level neighbours, restricted
// from the fine ghost cells the exchange filled
__global__ void k_fill_coarse(AmrArgs A, int emax) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)56 * A.nvar * emax;
  if (t >= per * A.nmb) return;
  const int m = (int)(t / per);
  long long r = t - (long long)m * per;
  const int n = (int)(r / ((long long)A.nvar * emax)); r -= (long long)n * A.nvar * emax;
  const int v = (int)(r / emax);
  const int e = (int)(r - (long long)v * emax);
  const int gs = A.nb[(long long)m * 56 + n];
  if (gs < 0) return;
  const int s = gs - A.gids;
  if (s < 0 || s >= A.nmb || A.lev[s] != A.lev[m]) return;
  const int o[3] = {A.tab.o[n][0], A.tab.o[n][1], A.tab.o[n][2]};
  const Box fb = recv_box(A.g, o, A.tab.o[n][3], A.tab.o[n][4], 0);
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = (fb.lo[d] + A.g.cis[d]) / 2;
    hi[d] = (fb.hi[d] + A.g.cis[d]) / 2;
  }
  const int ni = hi[0] - lo[0] + 1, nj = hi[1] - lo[1] + 1, nk = hi[2] - lo[2] + 1;
  if (e >= ni * nj * nk) return;
  const int i = lo[0] + e % ni, j = lo[1] + (e / ni) % nj, k = lo[2] + e / (ni * nj);
  A.ca[cidx(A, m, v, k, j, i)] = restrict8(A, m, v, k, j, i);
}

// the min-mod limited slope of ProlongCC (PROLONG_CC_SLOPE, src/mesh/prolongation.hpp:33)
__device__ __forceinline__ double mm_slope(double dl, double dr) {
  const double sl = (dl < 0.0) ? -1.0 : 1.0, sr = (dr < 0.0) ? -1.0 : 1.0;
  return 0.125 * (sl + sr) * fmin(fabs(dl), fabs(dr));
}

// 4. ProlongateCC: the fine ghost cells next to coarser neighbours from the coarse array
__global__ void k_prolong(AmrArgs A, int emax) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)56 * A.nvar * emax;
  if (t >= per * A.nmb) return;
  const int m = (int)(t / per);
  long long r = t - (long long)m * per;
  const int n = (int)(r / ((long long)A.nvar * emax)); r -= (long long)n * A.nvar * emax;
  const int v = (int)(r / emax);
  const int e = (int)(r - (long long)v * emax);
  const int gs = A.nb[(long long)m * 56 + n];
  if (gs < 0) return;
  const int s = gs - A.gids;
  if (s < 0 || s >= A.nmb || A.lev[s] >= A.lev[m]) return;
  const int o[3] = {A.tab.o[n][0], A.tab.o[n][1], A.tab.o[n][2]};
  const Box pb = recv_box(A.g, o, A.tab.o[n][3], A.tab.o[n][4], 3);
  const int ni = pb.hi[0] - pb.lo[0] + 1, nj = pb.hi[1] - pb.lo[1] + 1;
  const int nk = pb.hi[2] - pb.lo[2] + 1;
  if (e >= ni * nj * nk) return;
  const int i = pb.lo[0] + e % ni, j = pb.lo[1] + (e / ni) % nj, k = pb.lo[2] + e / (ni * nj);
  const double c = A.ca[cidx(A, m, v, k, j, i)];
  const double d1 = mm_slope(c - A.ca[cidx(A, m, v, k, j, i - 1)], A.ca[cidx(A, m, v, k, j, i + 1)] - c);
  const double d2 = mm_slope(c - A.ca[cidx(A, m, v, k, j - 1, i)], A.ca[cidx(A, m, v, k, j + 1, i)] - c);
  const double d3 = mm_slope(c - A.ca[cidx(A, m, v, k - 1, j, i)], A.ca[cidx(A, m, v, k + 1, j, i)] - c);
  const int fi = (i - A.g.cis[0]) * 2 + A.g.is[0];
  const int fj = (j - A.g.cis[1]) * 2 + A.g.is[1];
  const int fk = (k - A.g.cis[2]) * 2 + A.g.is[2];
  double *a = A.a;
  a[fidx(A, m, v, fk, fj, fi)] = c - d1 - d2 - d3;
  a[fidx(A, m, v, fk, fj, fi + 1)] = c + d1 - d2 - d3;
  a[fidx(A, m, v, fk, fj + 1, fi)] = c - d1 + d2 - d3;
  a[fidx(A, m, v, fk, fj + 1, fi + 1)] = c + d1 + d2 - d3;
  a[fidx(A, m, v, fk + 1, fj, fi)] = c - d1 - d2 + d3;
  a[fidx(A, m, v, fk + 1, fj, fi + 1)] = c + d1 - d2 + d3;
  a[fidx(A, m, v, fk + 1, fj + 1, fi)] = c - d1 + d2 + d3;
  a[fidx(A, m, v, fk + 1, fj + 1, fi + 1)] = c + d1 + d2 + d3;
}

}  // namespace

extern "C" {

long long dustb_ghost_copy_ml_bytes(const dustb_mesh *ms, int nvar) {
  if (!ms || nvar <= 0 || !ms->three_d) return -1;
  const Geo3 g = make_geo3(*ms);
  return (long long)ms->nmb * nvar * g.ccells * (long long)sizeof(double);
}

int dustb_ghost_copy_ml(const dustb_ctx *c, double *field, int nvar, double *coarse,
                        long long coarse_bytes, void *stream) {
  if (!c || !field || !coarse || nvar <= 0) return DUSTB_EINVAL;
  const dustb_mesh &ms = c->mesh;
  if (!ms.nghbr_ml || !ms.mb_lev || !ms.mb_size || ms.nmb <= 0) return DUSTB_EINVAL;
  // (3-D, even block sizes and ghost width, blocks of at least 2 ng cells; physical x3 faces
  // and shear-periodic faces are the single-level exchange's)
  if (!ms.three_d || ms.x3bc != DUSTB_X3_PERIODIC || ms.shear_x1) return DUSTB_EUNSUP;
  if ((ms.nx1 | ms.nx2 | ms.nx3 | ms.ng) & 1) return DUSTB_EUNSUP;
  if (ms.nx1 < 2 * ms.ng || ms.nx2 < 2 * ms.ng || ms.nx3 < 2 * ms.ng) return DUSTB_EUNSUP;
  if (coarse_bytes < dustb_ghost_copy_ml_bytes(&ms, nvar)) return DUSTB_ESCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  AmrArgs A;
  A.tab = make_slots();
  A.g = make_geo3(ms);
  A.nmb = ms.nmb; A.nvar = nvar; A.gids = ms.gids;
  A.nb = ms.nghbr_ml; A.lev = ms.mb_lev; A.mb = ms.mb_size;
  A.x1min = ms.x1min; A.x2min = ms.x2min; A.x3min = ms.x3min;
  A.a = field; A.ca = coarse;
  // the largest box of any slot and kind: a face strip of the fine array (nx^2 ng) bounds the
  // coarse boxes and the prolongation boxes
  int emax = 0;
  {
    const int ng = ms.ng, nx[3] = {ms.nx1, ms.nx2, ms.nx3};
    for (int d = 0; d < 3; ++d) {
      const int f = nx[(d + 1) % 3] * nx[(d + 2) % 3] * ng;
      if (f > emax) emax = f;
      const int cf = (nx[(d + 1) % 3] / 2 + ng) * (nx[(d + 2) % 3] / 2 + ng) * ng;
      if (cf > emax) emax = cf;
    }
  }
  cudaMemsetAsync(coarse, 0, (size_t)dustb_ghost_copy_ml_bytes(&ms, nvar), st);
  const long long nr = (long long)A.g.cnx[0] * A.g.cnx[1] * A.g.cnx[2] * nvar * ms.nmb;
  k_restrict<<<grid_for(nr), kThr, 0, st>>>(A);
  const long long ne = (long long)ms.nmb * 56 * nvar * emax;
  k_exchange<<<grid_for(ne), kThr, 0, st>>>(A, emax);
  k_fill_coarse<<<grid_for(ne), kThr, 0, st>>>(A, emax);
  k_prolong<<<grid_for(ne), kThr, 0, st>>>(A, emax);
  return dustb_host::launch_status("ghost_copy_ml");
}

}  // extern "C"
