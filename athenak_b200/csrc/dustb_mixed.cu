// dustb_mixed.cu -- the mixed-precision form of the imex2+ drag step.
//
// Particle shadow (structure of arrays, 4-byte words, two copies A and B): packed cell id
// (block, k, j, i), FP32 offsets inside the cell, velocity, velocity register, register
// displacement x1 - x in cells, drag rate, stopping time, mass, the cycle's drag factor
// a/(t_s + a) (formed in FP64), and the particle's row in the reference SoA.  The shadow is
// kept sorted by cell at every stage, so the particles of a tile of cells are one contiguous
// range, which the Tensor Memory Accelerator copies into shared memory with bulk copies.
// The mesh fields are the reference's FP64 arrays.
//
// One stage (the task order of src/dust/dust_tasks.cpp:56-107):
//   count     per particle: [stage 2: the stage-1 consistent dust kick] and the push of the
//             position; the new cell and a per-cell histogram
//   scan      of the histogram: the cell ranges of the new order
//   move      per particle: the whole push (register copy, velocity, position, the cell carry
//             that replaces SetNewPrtclGID), written to the particle's slot in the other copy
//   deposit   per CTA a tile of rows of cells of one plane, one thread per source cell; the
//             tile's particle range is bulk-copied (one copy per field) into shared memory in
//             passes; each thread walks its cell's particles: the 27 stencil weights,
//             [the gather of u* from the 27 cells around its cell, held in registers, the
//             kick] and the 27 x NC deposits accumulated in registers over all passes.  At the
//             end the threads of a row combine the x-offset contributions that land on the
//             same cell (warp shuffles) and add the sums to the FP64 field; cells beyond the
//             block go straight into the owning neighbour.  Three forms: Q/P + centre mass
//             (DepositDrag), the dc1 operator (PointOperatorParticles), the
//             gather-kick-deposit (GatherKickPMBR).
//   cells     the FP64 per-cell solves of dustb_fp64.cu
//   kick      [stage 2] the consistent dust kick (stage 1's is folded into stage 2's push)
// Weights, gathers and kicks are FP32; the drag factor a/(t_s + a) is formed in FP64; every
// deposit sum is added into FP64.  The kick deposits the velocity change the particle
// actually received (v_new - v in FP32).
#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "dustb_common.cuh"
#include "dustb_sort.cuh"

namespace dustb_cells {
void gas_rk(const dustb_ctx *c, double g0, double g1, cudaStream_t st);
void history(const dustb_ctx *c, double atw_dt, cudaStream_t st);
void history_field(const dustb_ctx *c, const double *f, double atw_dt, cudaStream_t st);
void dc_correct(const dustb_ctx *c, cudaStream_t st);
void consistent_gas(const dustb_ctx *c, double a_dt, cudaStream_t st);
void pmbr(const dustb_ctx *c, double a_dt, cudaStream_t st);
bool ctx_valid(const dustb_ctx *c);
}  // namespace dustb_cells

using namespace dustb;

namespace {

constexpr int kT = 256;
constexpr int kMaxTileThreads = 256;             // one thread per source cell of a tile
constexpr int kNF = 18;                          // FP32 arrays per copy

// FP32 array slots of a copy
enum { F_OX = 0, F_OY, F_OZ, F_VX, F_VY, F_VZ, F_AX, F_AY, F_AZ, F_WX, F_WY, F_WZ,
       F_RX, F_RY, F_RZ, F_TS, F_M, F_CC };

inline unsigned nblk(long long n) {
  long long b = (n + kT - 1) / kT;
  return (unsigned)(b < 1 ? 1 : b);
}
inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

struct PBuf {                    // one copy of the shadow
  int *cell, *pid;
  float *f[kNF];
};

// state kept in the workspace between calls: the stage-2 consistent dust kick of the last
// cycle is not applied to the shadow by that cycle; the next cycle's stage-1 push applies it
// (as stage 2's push applies stage 1's), and an export applies it to the rows it writes
struct MHead {
  int pending;                   // nonzero: the last cycle's consistent kick is pending
  int pad;
  double a_dt;                   // that cycle's a dt (the rate change is dv / a dt)
};

// the bins of the sort: one per active cell, then the edge bin (particles whose pc2 gather
// position lies beyond a physical x3 face or a shear-periodic x1 face), then the end
inline long long nbins(long long ncell) { return ncell + 2; }

struct MState {
  MHead *head;
  PBuf A, B;                     // A holds the shadow between cycles
  int *key;                      // new cell of each particle (count -> move)
  int *cstart, *cursor, *bsum;
  float4 *win;                   // 3-D: the gather window (k_gather_window)
  int *tile_order;               // the tiles heaviest first (the device work queue)
  int *qhead;                    // kQueues counters: tiles taken by each queued launch
};

// counters of the queued tile launches of a stage (Q/P, up to two operator sweeps, kick;
// the pc2 predictor and advance), cleared when the stage's queue is built
constexpr int kQueues = 8;
constexpr int kMaxLevels = 8;                    // refined meshes: levels above the root
enum { Q_QP = 0, Q_OP = 1, Q_KICK = 4, Q_PRED = 5, Q_ADV = 6 };

// cells of the gather window of a 3-D mesh: every block's active cells and one layer around
// them, (nx1 + 2)(nx2 + 2)(nx3 + 2) per block; 0 in 2-D (the 2-D tiles read the FP64 field)
long long nwin(const dustb_mesh &ms) {
  if (!ms.three_d) return 0;
  return (long long)ms.nmb * (ms.nx1 + 2) * (ms.nx2 + 2) * (ms.nx3 + 2);
}

struct Geo {
  int nmb, nx1, nx2, nx3, three_d, gids;
  int l1, l2, l3;              // log2 of nx1, nx2, nx3 when all are powers of two, else -1
  int n1, n2, n3, is, js, ks;
  long long vstride;           // cells of one variable of one block
  const int *nghbr;
  const double *mb;
  double dx[3], inv_dx[3], vol;
  int scheme;
  // 1: the tiles gather from and deposit into each block's own ghost cells (physical x3
  // faces or shear-periodic x1 faces; the FP64 ghost exchanges run around the tiles);
  // 0: cells beyond a block map to the owning neighbour's active cells
  int ghost;
  int x3bc;                    // DUSTB_X3_*
  // shear-periodic x1 faces of a 3-D shearing box (bvals_part.cpp:266-310)
  int sb_on, sb_nb2, sb_nb3;
  const int *sb_gid;
  double mx1min, mx1max, mx2min, mx3min, mly, mlz;   // mesh x1 range, lower y, z, y, z extents
  double shR;                  // fmod(q Omega Lx t, Ly) in cells of y
  int ncell;                   // active cells; key ncell = the edge bin (pc2 half step)
  int W1, W2, W3;              // 3-D: the gather window's cells per row, rows, planes of a block
  // refined meshes (ml = 1): every block's level (lev, by block, root_level first), the 56
  // neighbour slots, the root blocks per direction; dx and vol are the root level's, a block
  // of level l above the root has cells of dx / 2^l and volume vol / 8^l (exact: powers of
  // two; no per-level table, whose run-time index would make every thread copy this struct
  // out of the kernel's parameters); ml = 0 on a single-level mesh
  int ml, root;
  const int *lev, *nml;
  int nmbroot[3];
  __device__ int lv(int m) const {
    if (!ml) return 0;
    const int l = lev[m] - root;
    return l < 0 ? 0 : (l >= kMaxLevels ? kMaxLevels - 1 : l);
  }
  __device__ double dxm(int m, int a) const { return ml ? ldexp(dx[a], -lv(m)) : dx[a]; }
  __device__ double volm(int m) const { return ml ? ldexp(vol, -3 * lv(m)) : vol; }
  __device__ long long at(int m, int nvar, int v, int k, int j, int i) const {
    return (((long long)m * nvar + v) * vstride) + ((long long)k * n2 + j) * n1 + i;
  }
  // the owning block and active cell of block-local cell (k, j, i) of block m, which may
  // lie one cell outside the block (the same-level neighbour across the face); false if
  // no block owns it
  __device__ bool owner(int m, int &k, int &j, int &i, int &mo) const {
    const int o1 = (i < 0) ? -1 : ((i >= nx1) ? 1 : 0);
    const int o2 = (j < 0) ? -1 : ((j >= nx2) ? 1 : 0);
    const int o3 = (k < 0) ? -1 : ((k >= nx3) ? 1 : 0);
    if ((o1 | o2 | o3) == 0) { mo = m; return true; }
    mo = nghbr[(long long)m * 27 + dir_slot(o1, o2, o3)] - gids;
    i -= o1 * nx1; j -= o2 * nx2; k -= o3 * nx3;
    return mo >= 0 && mo < nmb;
  }
};

long long ncell_of(const dustb_mesh &ms) {
  return (long long)ms.nmb * ms.nx1 * (ms.multi_d ? ms.nx2 : 1) * (ms.three_d ? ms.nx3 : 1);
}

// workspace carving (the same order in every call)
bool carve(const dustb_mesh &ms, int n, void *ws, long long bytes, MState &S, long long *need) {
  const long long ncell = ncell_of(ms);
  const size_t N = (size_t)(n > 0 ? n : 1);
  size_t off = al256(sizeof(MHead));
  size_t o_buf[2][2 + kNF];
  for (int b = 0; b < 2; ++b)
    for (int f = 0; f < 2 + kNF; ++f) { o_buf[b][f] = off; off += al256(4 * N); }
  // the cell ranges: ncell cells, the edge bin (key ncell) and the end
  const size_t o_key = off; off += al256(4 * N);
  const size_t o_cs = off; off += al256(4 * (size_t)(ncell + 2));
  const size_t o_cur = off; off += al256(4 * (size_t)(ncell + 2));
  const size_t o_bs = off; off += al256(4 * (size_t)scan_bsum_ints(ncell + 2));
  const size_t o_win = off; off += al256(16 * (size_t)nwin(ms));
  // (tiles of one row each at most: the active rows of the mesh)
  const size_t o_ord = off; off += al256(4 * (size_t)(ncell / ms.nx1 + 1));
  const size_t o_qh = off; off += al256(4 * kQueues);
  if (need) *need = (long long)off;
  if (!ws || bytes < (long long)off) return false;
  char *b = (char *)ws;
  PBuf *bufs[2] = {&S.A, &S.B};
  for (int q = 0; q < 2; ++q) {
    bufs[q]->cell = (int *)(b + o_buf[q][0]);
    bufs[q]->pid = (int *)(b + o_buf[q][1]);
    for (int f = 0; f < kNF; ++f) bufs[q]->f[f] = (float *)(b + o_buf[q][2 + f]);
  }
  S.head = (MHead *)b;
  S.key = (int *)(b + o_key);
  S.cstart = (int *)(b + o_cs); S.cursor = (int *)(b + o_cur); S.bsum = (int *)(b + o_bs);
  S.win = (float4 *)(b + o_win);
  S.tile_order = (int *)(b + o_ord);
  S.qhead = (int *)(b + o_qh);
  return true;
}

Geo make_geo(const dustb_ctx *c, const dustb_mixed_params *mp) {
  const dustb_mesh &ms = c->mesh;
  Ind d = make_ind(ms);
  Geo G;
  G.nmb = ms.nmb; G.nx1 = d.nx1; G.nx2 = d.nx2; G.nx3 = d.nx3; G.three_d = ms.three_d;
  G.gids = ms.gids; G.n1 = d.n1; G.n2 = d.n2; G.n3 = d.n3; G.is = d.is; G.js = d.js; G.ks = d.ks;
  G.vstride = d.cells();
  G.nghbr = ms.nghbr; G.mb = ms.mb_size;
  auto lg = [](int n) { int l = 0; while ((1 << l) < n) ++l; return ((1 << l) == n) ? l : -1; };
  G.l1 = lg(G.nx1); G.l2 = lg(G.nx2); G.l3 = lg(G.nx3);
  if (G.l1 < 0 || G.l2 < 0 || G.l3 < 0) G.l1 = G.l2 = G.l3 = -1;
  for (int a = 0; a < 3; ++a) { G.dx[a] = mp->dx[a]; G.inv_dx[a] = 1.0 / mp->dx[a]; }
  // cell volume as the reference forms it: dx1 dx2 (dx3 in 3-D), dust_pm.cpp:253-254
  G.vol = mp->dx[0] * mp->dx[1] * (ms.three_d ? mp->dx[2] : 1.0);
  G.scheme = c->phys.scheme;
  G.x3bc = ms.three_d ? ms.x3bc : DUSTB_X3_PERIODIC;
  G.sb_on = (ms.shear_x1 && ms.three_d) ? 1 : 0;
  G.ghost = (G.x3bc != DUSTB_X3_PERIODIC || G.sb_on) ? 1 : 0;
  G.sb_nb2 = ms.sb_nb2; G.sb_nb3 = ms.sb_nb3; G.sb_gid = ms.sb_gid;
  G.mx1min = ms.x1min; G.mx1max = ms.x1max; G.mx2min = ms.x2min; G.mx3min = ms.x3min;
  G.mly = ms.x2max - ms.x2min; G.mlz = ms.x3max - ms.x3min;
  G.shR = 0.0;
  if (G.sb_on) {
    // the folded offset of the particles' crossing, as dustb_route forms it
    const double lx = ms.x1max - ms.x1min;
    const double ysh = fmod(c->phys.qshear * c->phys.omega0 * lx * ms.time, G.mly);
    G.shR = ysh * (double)((long long)ms.sb_nb2 * ms.nx2) / G.mly;
  }
  G.ncell = (int)ncell_of(ms);
  G.W1 = G.nx1 + 2; G.W2 = G.nx2 + 2; G.W3 = G.nx3 + 2;
  G.ml = (ms.nghbr_ml && ms.mb_lev) ? 1 : 0;
  G.root = mp->root_level;
  G.lev = ms.mb_lev; G.nml = ms.nghbr_ml;
  const double ext[3] = {ms.x1max - ms.x1min, ms.x2max - ms.x2min, ms.x3max - ms.x3min};
  const int nxs[3] = {d.nx1, d.nx2, d.nx3};
  for (int a = 0; a < 3; ++a) G.nmbroot[a] = (int)floor(ext[a] / (nxs[a] * mp->dx[a]) + 0.5);
  if (G.ml) G.ghost = 1;      // (the tiles on each block's own ghost cells, exchanged around them)
  return G;
}

__device__ __forceinline__ void decode(const Geo &G, int c, int &m, int &k, int &j, int &i) {
  if (G.l1 >= 0) {
    i = c & (G.nx1 - 1); c >>= G.l1;
    j = c & (G.nx2 - 1); c >>= G.l2;
    k = c & (G.nx3 - 1);
    m = c >> G.l3;
    return;
  }
  i = c % G.nx1; c /= G.nx1;
  j = c % G.nx2; c /= G.nx2;
  k = c % G.nx3;
  m = c / G.nx3;
}
__device__ __forceinline__ int encode(const Geo &G, int m, int k, int j, int i) {
  return ((m * G.nx3 + k) * G.nx2 + j) * G.nx1 + i;
}

// PMWeights in FP32 from the offset inside the cell (cell - ig of dust.hpp:1094-1096)
__device__ __forceinline__ void wts(int scheme, float o, float w[3]) {
  const float del = o - 0.5f;
  if (scheme == 2) {
    const float a = 0.5f - del, b = 0.5f + del;
    w[0] = 0.5f * a * a; w[1] = 0.75f - del * del; w[2] = 0.5f * b * b;
  } else if (scheme == 1) {
    w[0] = fmaxf(0.0f, -del); w[1] = 1.0f - fabsf(del); w[2] = fmaxf(0.0f, del);
  } else {
    w[0] = 0.0f; w[1] = 1.0f; w[2] = 0.0f;
  }
}

// lanes of a warp with the same key take consecutive slots from one atomic add on
// counter[key]; returns this lane's slot (keys of nearly cell-sorted particles come in runs)
__device__ __forceinline__ int warp_slot(int *counter, int key, unsigned act) {
  const unsigned peers = __match_any_sync(act, key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(&counter[key], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane) - 1u));
}
// the sum of v over the lanes of mask (FP64), in lane 0; mask is a prefix of the warp's lanes
// (the threads of a CTA whose size is not a multiple of 32): a lane adds only what a lane of
// the mask sent it
__device__ __forceinline__ double warp_sum(unsigned mask, double v) {
  const int nl = 32 - __clz(mask), lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double y = __shfl_down_sync(mask, v, o);
    if (lane + o < nl) v += y;
  }
  return v;
}
__device__ __forceinline__ void warp_count(int *counter, int key, unsigned act) {
  const unsigned peers = __match_any_sync(act, key);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counter[key], __popc(peers));
}

// ---- Tensor Memory Accelerator bulk copies and their barrier ------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n"
               ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// one contiguous global range into shared memory; both addresses and the size are
// multiples of 16 bytes (the caller rounds the particle range out to whole 16-byte groups)
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// one box of a 4-D tensor (the tensor map) into shared memory at dst (128-byte aligned); the
// innermost coordinate c0 is 0 (the box starts on a 16-byte boundary); no multicast
__device__ __forceinline__ void tensor_copy_4d(void *dst, const CUtensorMap *map, int c0, int c1,
                                               int c2, int c3, uint64_t *bar) {
  asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
               ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2),
                 "r"(c3), "r"(smem_u32(bar)) : "memory");
}
// orders this thread's earlier ordinary shared-memory accesses before later bulk copies
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the barrier's phase: at most 2^22 polls and 0.2 s (a copy of a pass takes
// microseconds); false (and the error bit) if it never completes.  Warp-uniform: the lanes of
// mask leave the loop together, so the warp is converged at the CTA barrier that follows (a
// CTA barrier assumes converged warps)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned *err,
                                          unsigned mask) {
  // (the clock is read every 1024 polls only: a completed copy costs no clock read)
  unsigned long long t0 = 0;
  for (int it = 0; it < (1 << 22); ++it) {
    if (__all_sync(mask, mbar_try_wait(bar, parity))) return true;
    if ((it & 1023) == 1023) {
      const unsigned long long t = global_ns();
      if (it == 1023) t0 = t;
      else if (__any_sync(mask, t - t0 > 200000000ull)) break;
    }
  }
  report(err, DUSTB_ERR_TIMEOUT);
  return false;
}

// ---- import / export / sort ----------------------------------------------------------------
// the reference rows of particle p into copy B (unsorted) and the histogram of its cells
__global__ void k_import(const double *pr, const int *pi, long long stride, int n, PBuf B,
                         int *count, Geo G, unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  auto R = [&](int r) { return pr[(long long)r * stride + p]; };
  int m = pi[(long long)DUSTB_PGID * stride + p] - G.gids;
  if (m < 0 || m >= G.nmb) { report(err, DUSTB_ERR_PGID); m = m < 0 ? 0 : G.nmb - 1; }
  const double *sz = G.mb + (long long)m * 9;
  const int nx[3] = {G.nx1, G.nx2, G.nx3};
  const double x[3] = {R(DUSTB_IPX), R(DUSTB_IPY), R(DUSTB_IPZ)};
  const double x1[3] = {R(DUSTB_IPX1), R(DUSTB_IPY1), R(DUSTB_IPZ1)};
  int ic[3] = {0, 0, 0};
  float of[3] = {0.5f, 0.5f, 0.5f}, dd[3] = {0.0f, 0.0f, 0.0f};
  for (int a = 0; a < (G.three_d ? 3 : 2); ++a) {
    const double cell = (x[a] - sz[a]) * ((double)nx[a] / (sz[3 + a] - sz[a]));
    int ig = (int)(cell + 1.0) - 1;
    if (ig < 0 || ig >= nx[a]) {
      // a position inside the block's box [min, max) whose cell rounded onto the upper face
      // (one ulp below it) is clamped into the last cell; one outside the box is an error
      if (!(x[a] >= sz[a] && x[a] < sz[3 + a])) report(err, DUSTB_ERR_HALO);
      ig = ig < 0 ? 0 : nx[a] - 1;
    }
    float fo = (float)(cell - (double)ig);
    if (!(fo >= 0.0f)) fo = 0.0f;
    if (fo >= 1.0f) fo = 0.99999994f;
    ic[a] = ig; of[a] = fo;
    dd[a] = (float)((x1[a] - x[a]) / G.dxm(m, a));
  }
  const int key = encode(G, m, ic[2], ic[1], ic[0]);
  B.cell[p] = key; B.pid[p] = p;
  B.f[F_OX][p] = of[0]; B.f[F_OY][p] = of[1]; B.f[F_OZ][p] = of[2];
  B.f[F_VX][p] = (float)R(DUSTB_IPVX); B.f[F_VY][p] = (float)R(DUSTB_IPVY); B.f[F_VZ][p] = (float)R(DUSTB_IPVZ);
  B.f[F_AX][p] = dd[0]; B.f[F_AY][p] = dd[1]; B.f[F_AZ][p] = dd[2];
  B.f[F_WX][p] = (float)R(DUSTB_IPVX1); B.f[F_WY][p] = (float)R(DUSTB_IPVY1); B.f[F_WZ][p] = (float)R(DUSTB_IPVZ1);
  B.f[F_RX][p] = (float)R(DUSTB_IPRX); B.f[F_RY][p] = (float)R(DUSTB_IPRY); B.f[F_RZ][p] = (float)R(DUSTB_IPRZ);
  B.f[F_TS][p] = (float)R(DUSTB_IPTS); B.f[F_M][p] = (float)R(DUSTB_IPM);
  B.f[F_CC][p] = 0.0f;
  warp_count(count, key, act);
}

__global__ void k_hist(const int *cell, int n, int *count) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (live) warp_count(count, cell[p], act);
}

// every particle of src into its slot of dst (cells as they are): the sort of the shadow
__global__ void k_sortmove(PBuf src, PBuf dst, int n, int *cursor) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  const int key = src.cell[p];
  const int q = warp_slot(cursor, key, act);
  dst.cell[q] = key; dst.pid[q] = src.pid[p];
#pragma unroll
  for (int f = 0; f < kNF; ++f) dst.f[f][q] = src.f[f][p];
}

// the shadow's particles into their reference rows; a pending consistent kick of the last
// cycle is applied to the exported velocities and rates in FP64 (the kick the gas's split
// gave them, exactly: the rows' momentum is the one the cycles exchanged)
__global__ void k_export(double *pr, int *pi, long long stride, int n, PBuf A, Geo G,
                         const double *res, const MHead *head) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int m, k, j, i;
  decode(G, A.cell[q], m, k, j, i);
  const int p = A.pid[q];
  double vel[3] = {A.f[F_VX][q], A.f[F_VY][q], A.f[F_VZ][q]};
  double rate[3] = {A.f[F_RX][q], A.f[F_RY][q], A.f[F_RZ][q]};
  if (res && head->pending && A.f[F_M][q] > 0.0f) {
    const long long b = G.at(m, 4, 0, k + G.ks, j + G.js, i + G.is);
    const double cj = (double)A.f[F_CC][q];
    for (int a = 0; a < 3; ++a) {
      const double d = __dmul_rn(cj, res[b + a * G.vstride]);
      vel[a] += d;
      rate[a] += d / head->a_dt;
    }
  }
  auto W = [&](int r, double v) { pr[(long long)r * stride + p] = v; };
  const double *sz = G.mb + (long long)m * 9;
  const double dxm[3] = {G.dxm(m, 0), G.dxm(m, 1), G.dxm(m, 2)};
  const double x = sz[X1MIN] + ((double)i + (double)A.f[F_OX][q]) * dxm[0];
  const double y = sz[X2MIN] + ((double)j + (double)A.f[F_OY][q]) * dxm[1];
  W(DUSTB_IPX, x); W(DUSTB_IPY, y);
  W(DUSTB_IPX1, x + (double)A.f[F_AX][q] * dxm[0]);
  W(DUSTB_IPY1, y + (double)A.f[F_AY][q] * dxm[1]);
  if (G.three_d) {
    const double z = sz[X3MIN] + ((double)k + (double)A.f[F_OZ][q]) * dxm[2];
    W(DUSTB_IPZ, z);
    W(DUSTB_IPZ1, z + (double)A.f[F_AZ][q] * dxm[2]);
  }
  W(DUSTB_IPVX, vel[0]); W(DUSTB_IPVY, vel[1]); W(DUSTB_IPVZ, vel[2]);
  W(DUSTB_IPVX1, A.f[F_WX][q]); W(DUSTB_IPVY1, A.f[F_WY][q]); W(DUSTB_IPVZ1, A.f[F_WZ][q]);
  W(DUSTB_IPRX, rate[0]); W(DUSTB_IPRY, rate[1]); W(DUSTB_IPRZ, rate[2]);
  // the mass as the mixed form carries it (FP32; 0 for a particle an outflow face removed),
  // so that the rows' momentum is the momentum the cycles exchanged with the gas
  W(DUSTB_IPM, (double)A.f[F_M][q]);
  pi[(long long)DUSTB_PGID * stride + p] = m + G.gids;
}

__global__ void k_copy_buf(PBuf src, PBuf dst, int n) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  dst.cell[p] = src.cell[p]; dst.pid[p] = src.pid[p];
#pragma unroll
  for (int f = 0; f < kNF; ++f) dst.f[f][p] = src.f[f][p];
}

// ---- push: count and move ------------------------------------------------------------------
// what a push does: an imex2+ stage (ExplicitPush imex), the pc2 half step to the gather
// position (dust_pc2_advance's x_h, y_h + q Omega x_h dt/2), or the pc2 move to the new
// position that the advance tile left as a displacement
enum { PK_IMEX = 0, PK_HALF = 1, PK_FULL = 2 };
// advance() flags
enum { AF_EDGE = 1, AF_REFLECT = 2, AF_REMOVED = 4 };

struct PushArgs {
  int kind;
  float gam0, gam1, atw_dt;
  float bdt;                  // beta*dt (velocity kick)
  float bdx[3];               // beta*dt/dx per axis (drift in cells; on a refined mesh the root
                              // level's, 2^l times it in a block of level l); pc2 half step: h/dx
  float gy;                   // pc2 half step: q Omega h / dy (the gather position's y shift
                              // per unit x of the half-step position)
  float sdy;                  // pc2 half step: q Omega dt / dy (the new y's shear drift)
  float shy;                  // imex: the stage's implicit shear shift sh / dy (the deposit and
                              // gather weights sit at y + sh x), 0 outside the 3-D shearing box
  double a_dt;                // imex: a dt; pc2 half step: h = dt/2
  int stage2;
  int sbox, strat;
  float q, om;
  double *x3rem;              // (mass, count) removed at outflow x3 faces (move only)
  // the consistent split's dust kick folded into the push: stage 2 applies stage 1's kick
  // (res = stage 1's dust residual); stage 1 applies the previous cycle's stage-2 kick when
  // head->pending is set (res = that residual)
  const double *res;
  MHead *head;
  int set_pending;            // stage 2: record this cycle's stage-2 kick as pending
  unsigned *err;
  // imex: the momentum ledger of the push.  The FP32 velocity a particle stores differs from
  // the FP64 value of the same update (the RK combination g0 v + g1 v1 of the gas's own FP64
  // coefficients, the folded consistent kick, the history term); m times the difference is
  // added to the gas momentum (u0, and at stage 1 also its register u1, which the push's
  // register copy pairs with) at the cell of each CTA's first particle.  Null: no ledger
  double *u0, *u1;
  int nvg;
  double g0, g1, atw;
  double inv_adt;              // 1/(a dt) (imex: the kick's share of the rate)
};

// dust_imex_point_consistent_dust of stage 1 (src/dust/dust_pm.cpp:686-696): the velocity
// change of the particle (c times the FP64 residual of its cell), explicitly rounded so that
// the count and the move kernel form bit-identical results
__device__ __forceinline__ void consistent_dv(const Geo &G, const PushArgs &P, float cc,
                                              int m, int k, int j, int i, double d[3]) {
  const long long b = G.at(m, 4, 0, k + G.ks, j + G.js, i + G.is);
  const double cj = (double)cc;
  d[0] = __dmul_rn(cj, P.res[b]);
  d[1] = __dmul_rn(cj, P.res[b + G.vstride]);
  d[2] = __dmul_rn(cj, P.res[b + 2 * G.vstride]);
}

// the y offset of the implicit stage's weight position y + sh x (ImplicitShearShift,
// src/dust/dust.hpp:1698-1702) in cells of the particle's own cell; explicitly rounded, so
// that the push and the tiles form it bit for bit alike
__device__ __forceinline__ float shifted_oy(const Geo &G, float shy, int m, int i, float ox,
                                            float oy) {
  const double *sz = G.mb + (long long)m * 9;
  const double x = __dadd_rn(sz[X1MIN], __dmul_rn(__dadd_rn((double)i, (double)ox), G.dx[0]));
  return __fadd_rn(oy, __fmul_rn(shy, __double2float_rn(x)));
}

// the new position in cell units, explicitly rounded so that count and move agree bit for
// bit.  imex: the drift of ExplicitPush (src/dust/dust_push.cpp:289-296),
// x <- x + gam1 (x1 - x) + beta dt xdot (gam0 + gam1 = 1); pc2 half step: x + h xdot with y
// shifted by q Omega x_h h (dust_push.cpp:132-140); pc2 move: x + the displacement the
// advance left in d1.  Then SetNewPrtclGID (src/bvals/bvals_part.cpp:159-429) as a cell
// carry: a physical x3 face reflects or removes the particle (bvals_part.cpp:167-197), a
// shear-periodic x1 face moves it to the face block on the other side at y -/+ the folded
// shear offset (bvals_part.cpp:266-310), any other face hands it to the neighbour across it
// (periodic images are neighbours).  The pc2 half step routes nothing: a gather position
// beyond a physical x3 face or a shear face sends the particle, unmoved, to the edge bin.

// the carried state of a particle that leaves its block
struct Carry {
  int key, m, k, j, i, flags;
  float o[3], d1[3];
};

// the face crossings, out of line (few particles take them; the common path stays small).
// (m, k, j, i) the old cell, (ni, nj, nk) the new block-local cell, on / dn the new offsets
// and displacement
__device__ __forceinline__ Carry cross_face(const Geo &G, const PushArgs &P, int m, int k, int j,
                                         int i, int ni, int nj, int nk, float on0, float on1,
                                         float on2, float dn0, float dn1, float dn2) {
  Carry C;
  C.flags = 0;
  const double *sz = G.mb + (long long)m * 9;
  const int o1 = (ni < 0) ? -1 : ((ni >= G.nx1) ? 1 : 0);
  const int o2 = (nj < 0) ? -1 : ((nj >= G.nx2) ? 1 : 0);
  int o3 = (nk < 0) ? -1 : ((nk >= G.nx3) ? 1 : 0);
  const bool x3face = o3 != 0 && G.x3bc != DUSTB_X3_PERIODIC &&
                      G.nghbr[(long long)m * 27 + dir_slot(0, 0, o3)] < 0;
  bool sbface = false;
  if (o1 != 0 && G.sb_on) {
    // this block's x1 face in the crossing direction lies on the mesh's (bvals_part.cpp:260-261)
    const double lx = sz[X1MAX] - sz[X1MIN];
    sbface = (o1 < 0) ? (sz[X1MIN] < G.mx1min + 0.5 * lx) : (sz[X1MAX] > G.mx1max - 0.5 * lx);
  }
  if (P.kind == PK_HALF && (x3face || sbface)) {
    // position and cell left as they were
    C.flags = AF_EDGE; C.key = G.ncell;
    C.m = m; C.k = k; C.j = j; C.i = i;
    C.o[0] = C.o[1] = C.o[2] = 0.0f; C.d1[0] = C.d1[1] = C.d1[2] = 0.0f;
    return C;
  }
  i = ni; j = nj; k = nk;
  float o[3] = {on0, on1, on2}, d1[3] = {dn0, dn1, dn2};
  if (x3face) {
    if (G.x3bc == DUSTB_X3_REFLECT) {
      // z <- 2 z_face - z: the offset mirrors, the register displacement changes sign (the
      // caller turns the z velocities); a particle exactly on the upper face stays just
      // below it, as the reference's snap
      float om_ = __fsub_rn(1.0f, o[2]);
      k = (o3 < 0) ? -k - 1 : 2 * G.nx3 - k - 1;
      if (om_ >= 1.0f) {
        if (o3 < 0) { om_ = 0.0f; ++k; } else { om_ = 0.99999994f; }
      }
      o[2] = om_;
      d1[2] = -d1[2];
      C.flags |= AF_REFLECT;
    } else {
      // outflow: removed (the caller zeroes mass and velocities), placed at the centre of the
      // block's edge cell with x1 = x
      k = (o3 < 0) ? 0 : G.nx3 - 1;
      o[2] = 0.5f;
      d1[0] = d1[1] = d1[2] = 0.0f;
      C.flags |= AF_REMOVED;
    }
    if (k < 0 || k >= G.nx3) { report(P.err, DUSTB_ERR_ROUTE); k = min(max(k, 0), G.nx3 - 1); }
    o3 = 0;
  }
  if ((o1 | o2 | o3) == 0) {
    // (nothing left to cross)
  } else if (sbface) {
    // the global y cell coordinate, shifted by -/+ the folded offset and wrapped; the face
    // block on the other side holding the new (y, z)
    const int N2 = G.sb_nb2 * G.nx2, N3 = G.sb_nb3 * G.nx3;
    const int b2 = (int)floor(__dadd_rn(__ddiv_rn(__dsub_rn(sz[X2MIN], G.mx2min),
                                                  __ddiv_rn(G.mly, (double)G.sb_nb2)), 0.5));
    const int b3 = (int)floor(__dadd_rn(__ddiv_rn(__dsub_rn(sz[X3MIN], G.mx3min),
                                                  __ddiv_rn(G.mlz, (double)G.sb_nb3)), 0.5));
    double Y = __dadd_rn((double)(b2 * G.nx2 + j), (double)o[1]);
    Y = (o1 < 0) ? __dsub_rn(Y, G.shR) : __dadd_rn(Y, G.shR);
    if (Y < 0.0) Y = __dadd_rn(Y, (double)N2);
    if (Y >= (double)N2) Y = __dsub_rn(Y, (double)N2);
    int Yc = (int)floor(Y);
    float oy = __double2float_rn(__dsub_rn(Y, (double)Yc));
    if (oy >= 1.0f) { oy = 0.0f; ++Yc; }
    Yc = (Yc % N2 + N2) % N2;
    const int Zc = ((b3 * G.nx3 + k) % N3 + N3) % N3;   // (x3 periodic here, or k inside)
    const int c2 = Yc / G.nx2, c3 = Zc / G.nx3;
    const int g = G.sb_gid[((long long)(o1 < 0 ? 1 : 0) * G.sb_nb3 + c3) * G.sb_nb2 + c2] - G.gids;
    if (g < 0 || g >= G.nmb) {
      report(P.err, DUSTB_ERR_NGHBR);
    } else {
      m = g; i -= o1 * G.nx1; j = Yc - c2 * G.nx2; k = Zc - c3 * G.nx3; o[1] = oy;
    }
  } else {
    const int g = G.nghbr[(long long)m * 27 + dir_slot(o1, o2, o3)] - G.gids;
    if (g < 0 || g >= G.nmb) {
      report(P.err, DUSTB_ERR_NGHBR);
    } else {
      m = g; i -= o1 * G.nx1; j -= o2 * G.nx2; k -= o3 * G.nx3;
    }
  }
  if (i < 0 || i >= G.nx1 || j < 0 || j >= G.nx2 || k < 0 || k >= G.nx3) {
    report(P.err, DUSTB_ERR_ROUTE);
    i = min(max(i, 0), G.nx1 - 1); j = min(max(j, 0), G.nx2 - 1); k = min(max(k, 0), G.nx3 - 1);
  }
  C.m = m; C.k = k; C.j = j; C.i = i;
  for (int a = 0; a < 3; ++a) { C.o[a] = o[a]; C.d1[a] = d1[a]; }
  C.key = encode(G, m, k, j, i);
  return C;
}

// A particle leaving block m of a refined (periodic) mesh at block-local cell (ni, nj, nk) with
// offsets o and register displacement d1 (cells of m's level): the block that holds it (the
// slot search of SetNewPrtclGID, ml_route_slot, with the halves the new position lies in) and
// its cell, offset and displacement in that block's cells.  The position is carried as cells
// of the mesh at m's level (the block's logical location times its cells plus the local
// coordinate), scaled by 2 or 1/2 to the neighbour's level (exact in FP64), wrapped across
// the periodic faces and taken relative to the neighbour's origin; the displacement scales the
// same way.  Count and move take the same steps, so they agree bit for bit.  Values in and
// out, no addresses: a caller's variable whose address reached this (not inlined) function
// would live in local memory on every path of the push.
struct MlCarry {
  int m, k, j, i, key;
  float o[3], d1[3];
};
__device__ __noinline__ MlCarry ml_carry(const Geo &G, const PushArgs &P, int m_in, int ni,
                                         int nj, int nk, float o0, float o1, float o2,
                                         float e0, float e1, float e2) {
  MlCarry r;
  int &m = r.m, &k = r.k, &j = r.j, &i = r.i;
  float *o = r.o, *d1 = r.d1;
  m = m_in;
  o[0] = o0; o[1] = o1; o[2] = o2;
  d1[0] = e0; d1[1] = e1; d1[2] = e2;
  const int nxs[3] = {G.nx1, G.nx2, G.nx3};
  const int nn[3] = {ni, nj, nk};
  int oc[3], f[3];
  for (int a = 0; a < 3; ++a) {
    oc[a] = (nn[a] < 0) ? -1 : ((nn[a] >= nxs[a]) ? 1 : 0);
    f[a] = (oc[a] != 0) ? (oc[a] > 0 ? 1 : 0) : (nn[a] >= nxs[a] / 2 ? 1 : 0);
  }
  const double *mbm = G.mb + (long long)m * 9;
  const int s = ml_route_slot(G.nml + (long long)m * 56, G.lev, G.gids, G.lev[m], mbm, G.mx1min,
                              G.mx2min, G.mx3min, oc[0], oc[1], oc[2], f[0], f[1], f[2]);
  const int t = (s < 0) ? -1 : G.nml[(long long)m * 56 + s] - G.gids;
  if (t < 0 || t >= G.nmb) {
    report(P.err, DUSTB_ERR_NGHBR);
    i = min(max(ni, 0), G.nx1 - 1); j = min(max(nj, 0), G.nx2 - 1); k = min(max(nk, 0), G.nx3 - 1);
    for (int a = 0; a < 3; ++a) o[a] = min(max(o[a], 0.0f), 0.99999994f);
    r.key = encode(G, m, k, j, i);
    return r;
  }
  const int rel = G.lev[t] - G.lev[m];
  const double sc = (rel > 0) ? 2.0 : ((rel < 0) ? 0.5 : 1.0);
  const double *mbt = G.mb + (long long)t * 9;
  const double mlo[3] = {G.mx1min, G.mx2min, G.mx3min};
  int c[3];
  for (int a = 0; a < 3; ++a) {
    const double lm = mbm[3 + a] - mbm[a], lt = mbt[3 + a] - mbt[a];
    const double lxm = floor((mbm[a] - mlo[a]) / lm + 0.5), lxt = floor((mbt[a] - mlo[a]) / lt + 0.5);
    // the mesh's extent in cells of the neighbour's level
    const double nt = (double)G.nmbroot[a] * nxs[a] * (double)(1 << (G.lev[t] - G.root));
    double x = (lxm * nxs[a] + (double)nn[a] + (double)o[a]) * sc;
    if (x < 0.0) x += nt; else if (x >= nt) x -= nt;
    const double loc = x - lxt * nxs[a];
    int ci = (int)floor(loc);
    float fo = (float)(loc - (double)ci);
    if (fo >= 1.0f) { fo = 0.0f; ++ci; }
    if (ci < 0 || ci >= nxs[a]) { report(P.err, DUSTB_ERR_ROUTE); ci = min(max(ci, 0), nxs[a] - 1); }
    c[a] = ci;
    o[a] = fo;
    d1[a] = (float)((double)d1[a] * sc);
  }
  m = t; i = c[0]; j = c[1]; k = c[2];
  r.key = encode(G, m, k, j, i);
  return r;
}

template <int KIND, int SP>
__device__ __forceinline__ int advance_carry(const Geo &G, const PushArgs &P, int &m, int &k,
                                             int &j, int &i, float o[3], float d1[3],
                                             const float v[3], int &flags, float hpos[2]) {
  flags = 0;
  hpos[0] = hpos[1] = 0.0f;
  float xsh = 0.0f;
  if (KIND != PK_FULL && P.sbox && G.three_d) {
    const double *sz = G.mb + (long long)m * 9;
    const double x = __dadd_rn(sz[X1MIN], __dmul_rn(__dadd_rn((double)i, (double)o[0]), G.dx[0]));
    xsh = __fmul_rn(__fmul_rn(P.q, P.om), __double2float_rn(x));
  }
  const float xdot[3] = {v[0], __fsub_rn(v[1], xsh), v[2]};
  const int nax = G.three_d ? 3 : 2;
  float on[3] = {o[0], o[1], o[2]}, dn[3] = {d1[0], d1[1], d1[2]};
  int c[3] = {0, 0, 0};
  for (int a = 0; a < nax; ++a) {
    const float bdx = (SP == 2) ? ldexpf(P.bdx[a], G.lv(m)) : P.bdx[a];
    float s = __fmaf_rn(bdx, xdot[a], __fmul_rn(P.gam1, d1[a]));
    // (the gather position's y: + q Omega x_h h, x_h the half-step x in this block's frame)
    if (KIND == PK_HALF && a == 1 && P.gy != 0.0f) s = __fmaf_rn(P.gy, hpos[0], s);
    on[a] = __fadd_rn(on[a], s);
    dn[a] = __fsub_rn(dn[a], s);
    if (KIND == PK_HALF && a != 1) {
      // the half-step x and z in this block's frame (before any carry or periodic wrap)
      const double *sz = G.mb + (long long)m * 9;
      const double x = __dadd_rn(sz[a == 0 ? X1MIN : X3MIN],
                                 __dmul_rn(__dadd_rn((double)(a == 0 ? i : k), (double)on[a]), G.dx[a]));
      hpos[a == 0 ? 0 : 1] = __double2float_rn(x);
    }
    int ci = (int)floorf(on[a]);
    on[a] = __fsub_rn(on[a], (float)ci);
    if (on[a] >= 1.0f) { on[a] = __fsub_rn(on[a], 1.0f); ++ci; }
    c[a] = ci;
  }
  const int ni = i + c[0], nj = j + c[1], nk = k + c[2];
  if ((unsigned)ni < (unsigned)G.nx1 && (unsigned)nj < (unsigned)G.nx2 &&
      (unsigned)nk < (unsigned)G.nx3) {
    i = ni; j = nj; k = nk;
    for (int a = 0; a < 3; ++a) { o[a] = on[a]; d1[a] = dn[a]; }
    return encode(G, m, k, j, i);
  }
  if constexpr (SP == 2) {
    const MlCarry r = ml_carry(G, P, m, ni, nj, nk, on[0], on[1], on[2], dn[0], dn[1], dn[2]);
    m = r.m; k = r.k; j = r.j; i = r.i;
    for (int a = 0; a < 3; ++a) { o[a] = r.o[a]; d1[a] = r.d1[a]; }
    return r.key;
  }
  if (SP == 0) {
    // a periodic mesh: the neighbour across the face (periodic images are neighbours)
    const int o1 = (ni < 0) ? -1 : ((ni >= G.nx1) ? 1 : 0);
    const int o2 = (nj < 0) ? -1 : ((nj >= G.nx2) ? 1 : 0);
    const int o3 = (nk < 0) ? -1 : ((nk >= G.nx3) ? 1 : 0);
    i = ni; j = nj; k = nk;
    for (int a = 0; a < 3; ++a) { o[a] = on[a]; d1[a] = dn[a]; }
    const int g = G.nghbr[(long long)m * 27 + dir_slot(o1, o2, o3)] - G.gids;
    if (g < 0 || g >= G.nmb) {
      report(P.err, DUSTB_ERR_NGHBR);
    } else {
      m = g; i -= o1 * G.nx1; j -= o2 * G.nx2; k -= o3 * G.nx3;
    }
    if (i < 0 || i >= G.nx1 || j < 0 || j >= G.nx2 || k < 0 || k >= G.nx3) {
      report(P.err, DUSTB_ERR_ROUTE);
      i = min(max(i, 0), G.nx1 - 1); j = min(max(j, 0), G.nx2 - 1); k = min(max(k, 0), G.nx3 - 1);
    }
    return encode(G, m, k, j, i);
  }
  const Carry C = cross_face(G, P, m, k, j, i, ni, nj, nk, on[0], on[1], on[2], dn[0], dn[1], dn[2]);
  flags = C.flags;
  if (!(flags & AF_EDGE)) {
    m = C.m; k = C.k; j = C.j; i = C.i;
    for (int a = 0; a < 3; ++a) { o[a] = C.o[a]; d1[a] = C.d1[a]; }
  }
  return C.key;
}

// the push of advance_carry; an imex stage with an implicit shear shift sends a particle
// whose shifted weight position lies in another cell to the edge bin (its true, new cell is
// kept; per-particle kernels deposit and gather it)
template <int KIND, int SP>
__device__ __forceinline__ int advance(const Geo &G, const PushArgs &P, int &m, int &k, int &j,
                                       int &i, float o[3], float d1[3], const float v[3],
                                       int &flags, float hpos[2]) {
  const int key = advance_carry<KIND, SP>(G, P, m, k, j, i, o, d1, v, flags, hpos);
  if (KIND == PK_IMEX && P.shy != 0.0f && !(flags & AF_EDGE)) {
    const float oy = shifted_oy(G, P.shy, m, i, o[0], o[1]);
    if (oy < 0.0f || oy >= 1.0f) { flags |= AF_EDGE; return G.ncell; }
  }
  return key;
}

// count: the new cell of every particle and the per-cell histogram
// SP: 0 a periodic single-level mesh, 1 physical x3 or shear-periodic x1 faces, 2 a refined
// (periodic) mesh
template <int KIND, int SP>
__global__ void __launch_bounds__(kT) k_count(PBuf S, int *key_out, int *count,
                                              const __grid_constant__ Geo G, int n,
                                              const __grid_constant__ PushArgs P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  int m, k, j, i;
  decode(G, S.cell[p], m, k, j, i);
  float o[3] = {S.f[F_OX][p], S.f[F_OY][p], S.f[F_OZ][p]};
  float v[3] = {S.f[F_VX][p], S.f[F_VY][p], S.f[F_VZ][p]};
  float d1[3] = {0.0f, 0.0f, 0.0f};
  if (P.stage2 || KIND == PK_FULL) { d1[0] = S.f[F_AX][p]; d1[1] = S.f[F_AY][p]; d1[2] = S.f[F_AZ][p]; }
  if (KIND != PK_FULL && P.res && (P.stage2 || P.head->pending) && S.f[F_M][p] > 0.0f) {
    double d[3];
    consistent_dv(G, P, S.f[F_CC][p], m, k, j, i, d);
    for (int a = 0; a < 3; ++a) v[a] = __fadd_rn(v[a], __double2float_rn(d[a]));
  }
  int flags;
  float hpos[2];
  const int key = advance<KIND, SP>(G, P, m, k, j, i, o, d1, v, flags, hpos);
  key_out[p] = key;
  warp_count(count, key, act);
  if (P.set_pending && p == 0) { P.head->a_dt = P.a_dt; P.head->pending = 1; }
}

// move: the whole push of every particle, written to its slot in dst; comp receives
// m (v_FP64 - v_stored) of the imex ledger
template <int KIND, int SP>
__device__ __forceinline__ void move_particle(const PBuf &S, const PBuf &D, const int *key_in,
                                              int *cursor, const Geo &G, const PushArgs &P,
                                              int p, unsigned act, double comp[3]) {
  const int key = key_in[p];
  // the source copy is only read here: its loads go through the read-only path and are all
  // issued before the slot's atomic, whose round trip then overlaps theirs
  const float *const *sf = S.f;
  int m, k, j, i;
  decode(G, __ldg(S.cell + p), m, k, j, i);
  float o[3] = {__ldg(sf[F_OX] + p), __ldg(sf[F_OY] + p), __ldg(sf[F_OZ] + p)};
  float v[3] = {__ldg(sf[F_VX] + p), __ldg(sf[F_VY] + p), __ldg(sf[F_VZ] + p)};
  const float ts = __ldg(sf[F_TS] + p);
  float mass = __ldg(sf[F_M] + p);
  const int pid = __ldg(S.pid + p);
  float v1[3], d1[3], r[3] = {0.0f, 0.0f, 0.0f}, cc;
  const bool kick = KIND != PK_FULL && P.res && (P.stage2 || P.head->pending);
  if (KIND == PK_FULL || P.stage2) {
    // pc2: the advance left the new velocity, the rate and the displacement to the new
    // position; the register velocity is v0.  imex stage 2: the stage registers and rates
    v1[0] = __ldg(sf[F_WX] + p); v1[1] = __ldg(sf[F_WY] + p); v1[2] = __ldg(sf[F_WZ] + p);
    d1[0] = __ldg(sf[F_AX] + p); d1[1] = __ldg(sf[F_AY] + p); d1[2] = __ldg(sf[F_AZ] + p);
    r[0] = __ldg(sf[F_RX] + p); r[1] = __ldg(sf[F_RY] + p); r[2] = __ldg(sf[F_RZ] + p);
  }
  // (imex stage 1 and the pc2 half step: the rates are not read; every kick rewrites them)
  cc = (KIND == PK_FULL || P.stage2 || kick) ? __ldg(sf[F_CC] + p) : 0.0f;
  const int q = warp_slot(cursor, key, act);
  // (the ledger's inputs: the velocity and rate before the folded kick, the kick in FP64)
  const float vb[3] = {v[0], v[1], v[2]}, rb[3] = {r[0], r[1], r[2]};
  double dk[3] = {0.0, 0.0, 0.0};
  if (KIND != PK_FULL) {
    if (kick && mass > 0.0f) {
      double d[3];
      consistent_dv(G, P, cc, m, k, j, i, d);
      for (int a = 0; a < 3; ++a) {
        v[a] = __fadd_rn(v[a], __double2float_rn(d[a]));
        // (imex: the rate takes the kick in the FP32 update below, the only reader of r)
        if (KIND != PK_IMEX) r[a] += (float)(d[a] / P.a_dt);
        dk[a] = d[a];
      }
    }
    if (!P.stage2) {
      // FirstTwoImpRK: (x1, v1) <- (x, v); the drag factor of the cycle, formed in FP64
      // (imex: a/(t_s + a); pc2: h/(t_s + h))
      v1[0] = v[0]; v1[1] = v[1]; v1[2] = v[2];
      d1[0] = d1[1] = d1[2] = 0.0f;
      cc = (float)(P.a_dt / ((double)ts + P.a_dt));
    }
  }
  float nv[3] = {v[0], v[1], v[2]};
  if (KIND == PK_IMEX) {
    // ExplicitPush imex (src/dust/dust_push.cpp:262-288): forces from the pre-stage velocity
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (P.sbox) {
      if (G.three_d) {
        fx = 2.0f * P.om * v[1];
        fy = -(2.0f - P.q) * P.om * v[0];
        if (P.strat) {
          const double *sz = G.mb + (long long)m * 9;
          fz = -(P.om * P.om) * (float)(sz[X3MIN] + ((double)k + o[2]) * G.dx[2]);
        }
      } else {
        fx = 2.0f * P.om * v[2];
        fz = -(2.0f - P.q) * P.om * v[0];
      }
    }
    if (!(P.u0 && mass > 0.0f)) {
      // the FP32 update (no ledger)
      if (kick && mass > 0.0f)
        for (int a = 0; a < 3; ++a) r[a] += (float)(dk[a] * P.inv_adt);
      const float atw = P.stage2 ? P.atw_dt : 0.0f;
      nv[0] = P.gam0 * v[0] + P.gam1 * v1[0] + P.bdt * fx + atw * r[0];
      nv[1] = P.gam0 * v[1] + P.gam1 * v1[1] + P.bdt * fy + atw * r[1];
      nv[2] = P.gam0 * v[2] + P.gam1 * v1[2] + P.bdt * fz + atw * r[2];
    } else {
      // the same update in FP64 from the stored inputs (the gas's coefficients, the exact kick
      // -- c times the FP64 residual -- in the velocity and, over a dt, in the rate), stored
      // rounded once to FP32 (half an ulp, where the FP32 chain leaves up to two); the ledger
      // takes m times what the rounding left out.  Stage 1 (g0 = 1, g1 = 0, no history term)
      // has only the kick, and its register copy is the kicked velocity rounded the same way
      const float fv[3] = {P.bdt * fx, P.bdt * fy, P.bdt * fz};
      const double mm = (double)mass;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double base = (double)vb[a] + dk[a];
        double want = base;
        if (P.stage2)
          want = fma(P.atw, fma(dk[a], P.inv_adt, (double)rb[a]), fma(P.g1, (double)v1[a], P.g0 * base));
        else
          v1[a] = __double2float_rn(base);
        if (P.sbox) want += (double)fv[a];
        nv[a] = __double2float_rn(want);
        comp[a] = mm * (want - (double)nv[a]);
      }
    }
  }
  int flags;
  float hpos[2];
  const int key2 = advance<KIND, SP>(G, P, m, k, j, i, o, d1, v, flags, hpos);
  if (key2 != key) report(P.err, DUSTB_ERR_WINDOW);   // count and move disagree: never expected
  if (KIND == PK_HALF && P.sbox && G.three_d && !(flags & AF_EDGE)) {
    // the shear drift -q Omega x_h dt of the new y goes into the displacement now, and z_h
    // (for the vertical gravity) into the rate slot, while x_h and z_h are known in the
    // frame of the particle's own block (the gather position may be a periodic image)
    d1[1] = __fsub_rn(d1[1], __fmul_rn(P.sdy, hpos[0]));
    r[2] = hpos[1];
  }
  if (flags & AF_REFLECT) { nv[2] = -nv[2]; v1[2] = -v1[2]; }
  if (flags & AF_REMOVED) {
    if (P.x3rem) { atomicAdd(&P.x3rem[0], (double)mass); atomicAdd(&P.x3rem[1], 1.0); }
    mass = 0.0f;
    for (int a = 0; a < 3; ++a) { nv[a] = 0.0f; v1[a] = 0.0f; }
  }
  // (an edge particle keeps its cell; its slot is in the edge bin)
  D.cell[q] = (flags & AF_EDGE) ? encode(G, m, k, j, i) : key;
  D.pid[q] = pid;
  D.f[F_OX][q] = o[0]; D.f[F_OY][q] = o[1]; D.f[F_OZ][q] = o[2];
  D.f[F_VX][q] = nv[0]; D.f[F_VY][q] = nv[1]; D.f[F_VZ][q] = nv[2];
  D.f[F_AX][q] = d1[0]; D.f[F_AY][q] = d1[1]; D.f[F_AZ][q] = d1[2];
  D.f[F_WX][q] = v1[0]; D.f[F_WY][q] = v1[1]; D.f[F_WZ][q] = v1[2];
  // (imex, pc2 half step: no rates, the stage's kick or advance writes every particle's;
  // the half step of a 3-D shearing box keeps z_h in the z rate until the advance)
  if (KIND == PK_FULL) { D.f[F_RX][q] = r[0]; D.f[F_RY][q] = r[1]; D.f[F_RZ][q] = r[2]; }
  else if (KIND == PK_HALF && P.sbox && G.three_d) D.f[F_RZ][q] = r[2];
  D.f[F_TS][q] = ts; D.f[F_M][q] = mass; D.f[F_CC][q] = cc;
}

template <int KIND, int SP>
__global__ void __launch_bounds__(kT) k_move(PBuf S, PBuf D, const int *key_in, int *cursor,
                                             const __grid_constant__ Geo G, int n,
                                             const __grid_constant__ PushArgs P) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  double comp[3] = {0.0, 0.0, 0.0};
  if (live) move_particle<KIND, SP>(S, D, key_in, cursor, G, P, p, act, comp);
  if constexpr (KIND == PK_IMEX) {
    if (!P.u0) return;
    // the CTA's ledger, added to the gas at its first particle's (old) cell: the particles of
    // a CTA are consecutive in cell order.  Staged in shared memory and summed by three warps,
    // one per direction (a warp sum per warp would cost every thread the shuffles)
    __shared__ double s_comp[3][kT];
#pragma unroll
    for (int a = 0; a < 3; ++a) s_comp[a][threadIdx.x] = comp[a];
    __syncthreads();
    const int a = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (a < 3) {
      double t = 0.0;
      for (int x = lane; x < kT; x += 32) t += s_comp[a][x];
      t = warp_sum(0xffffffffu, t);
      if (lane == 0 && t != 0.0) {
        int m, k, j, i;
        decode(G, S.cell[blockIdx.x * kT], m, k, j, i);
        const double vinv = 1.0 / ((SP == 2) ? G.volm(m) : G.vol);
        const long long at = G.at(m, P.nvg, 1 + a, G.ks + k, G.js + j, G.is + i);
        atomicAdd(&P.u0[at], t * vinv);
        if (!P.stage2 && P.u1) atomicAdd(&P.u1[at], t * vinv);
      }
    }
  }
}

// ---- tile deposit kernels -------------------------------------------------------------------
// Q/P + centre mass (imex), the dc1 operator, the gather-kick-deposit (imex), the pc2
// predictor, the pc2 advance
enum { MODE_QP = 0, MODE_OP = 1, MODE_KICK = 2, MODE_PRED = 3, MODE_ADV = 4 };

// the pc2 constants of a cycle in FP32 (dust_push.cpp:132-245)
struct Pc2Args {
  float dt, h;
  float cxy, cyx;              // 3-D shearing box: 2 h Omega, h (2 - q) Omega (x-z: cxz, czx)
  float qom;                   // q Omega (the shear drift of y)
  float hom2;                  // h Omega^2 (stratified vertical gravity)
  float haphi;                 // h const_accel_phi (2-D x-z shearing box)
  float hdx[3];                // h / dx per axis (the half step in cells)
  float gy;                    // q Omega h / dy (the gather position's y shift per unit x)
  int sbox, strat;
};

struct TileArgs {
  int tj, chunk, tpp;          // rows per tile, buffer columns, tiles per (block, plane)
  double a_dt;
  const int *cstart;           // cell -> particle ranges of the sorted shadow
  const double *gfield;        // gather field (3 vars): operator, kick, predictor, advance
  const float4 *win4;          // 3-D: the gather field's window (k_gather_window)
  double *dfield;              // deposit field (the predictor: qdep's variable 1)
  int dnvar;
  double *res;                 // MODE_QP: resid, the centre mass goes to var 3
  double *hfield;              // MODE_KICK: the rate's rounding for the history term (or null)
  int deposit;                 // 0: kick or advance only (no back-reaction)
  int ledger;                  // MODE_KICK: keep the tile's momentum ledger
  float shy;                   // imex: the stage's implicit shear shift sh / dy (0: none)
  int probe_timeout;           // test hook: tile 0 never issues its first copy
  // the device work queue of a persistent launch: the tiles in the order to take them
  // (heaviest first) and the launch's counter of tiles taken; order null: one CTA per tile
  const int *order;
  int *qhead;
  int ntiles;
  Pc2Args pc;
  unsigned *err;
};

// shared rows of a tile pass: the copied fields, then (operator, kick) the per-particle
// values of the gather phase in rows 5..7
constexpr int kTileRows = 8;

// the index of variable 0 of block-local cell (kk, jj, ii) of block m in a field of nvar
// variables, or -1 if no block owns it; a cell one beyond the block maps to the owning
// neighbour's active cell (the ghost exchanges folded into the index)
// GH: bit 0 ghost mode; (tiles) bit 1 the imex stage's implicit shear shift, compiled in only
// where it is used
template <int GH>
__device__ __forceinline__ long long cell_at(const Geo &G, int m, int nvar, int kk, int jj, int ii) {
  // (ghost mode: the block's own cell, ghost cells included; the window reaches one cell
  // beyond the block and every block has at least two ghost layers)
  if (GH & 1) return G.at(m, nvar, 0, G.ks + kk, G.js + jj, G.is + ii);
  int mo;
  if (!G.owner(m, kk, jj, ii, mo)) return -1;
  return G.at(mo, nvar, 0, G.ks + kk, G.js + jj, G.is + ii);
}
__device__ __forceinline__ float2 dup(float x) { return make_float2(x, x); }

// The 3-D tiles' gather window: the gather field (3 FP64 variables) on every block's active
// cells and one layer of cells around them, rounded to FP32 (x, y, z, 0) per cell, cell
// (k, j, i) at window index (k + 1, j + 1, i + 1).  GH = 1: the cells around a block are its
// own ghost cells (the FP64 copy exchange fills them); GH = 0: the owning neighbour's active
// cells (the exchange folded into the read).  Written once per gather, it replaces the 27
// owner lookups and 81 FP64 loads each tile thread made per cell.
template <int GH>
__global__ void __launch_bounds__(256) k_gather_window(const double *f, float4 *win, Geo G) {
  const long long total = (long long)G.W1 * G.W2 * G.W3 * G.nmb;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    long long r = idx;
    const int ii = (int)(r % G.W1); r /= G.W1;
    const int jj = (int)(r % G.W2); r /= G.W2;
    const int kk = (int)(r % G.W3);
    const int m = (int)(r / G.W3);
    const long long at = cell_at<GH>(G, m, 3, kk - 1, jj - 1, ii - 1);
    float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (at >= 0)
      v = make_float4((float)f[at], (float)f[at + G.vstride], (float)f[at + 2 * G.vstride], 0.0f);
    win[idx] = v;
  }
}

// the 27-point sums of one source cell's particles: values 0, 1 as a packed pair; values 2, 3
// as a pair (Q/P) or value 2 alone (operator, kick)
// (four values: Q/P and the predictor)
template <int MODE>
struct FourValues { static constexpr bool value = (MODE == MODE_QP || MODE == MODE_PRED); };

template <int MODE, int D3>
struct CellSums {
  static constexpr int WK = D3 ? 3 : 1;
  static constexpr bool V4 = FourValues<MODE>::value;
  float2 a01[WK][3][3], a23[WK][3][3];
  float a2[WK][3][3];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int c = 0; c < WK; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          a01[c][b][a] = make_float2(0.0f, 0.0f);
          if (V4) a23[c][b][a] = make_float2(0.0f, 0.0f);
          else a2[c][b][a] = 0.0f;
        }
  }
  __device__ __forceinline__ float val(int c, int b, int a, int q) const {
    return q == 0 ? a01[c][b][a].x : q == 1 ? a01[c][b][a].y
         : (V4 ? (q == 2 ? a23[c][b][a].x : a23[c][b][a].y) : a2[c][b][a]);
  }
  // sum_cba += wz_c wy_b (wx_a q): the x weights folded into the values first
  __device__ __forceinline__ void add(const float wx[3], const float wy[3], const float wz[3],
                                      float2 q01, float2 q23) {
    float2 s01[3], s23[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      s01[a] = __fmul2_rn(dup(wx[a]), q01);
      if (V4) s23[a] = __fmul2_rn(dup(wx[a]), q23);
      else s23[a].x = wx[a] * q23.x;
    }
#pragma unroll
    for (int c = 0; c < WK; ++c) {
      const float wzc = D3 ? wz[c] : 1.0f;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const float wzy = wzc * wy[b];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          a01[c][b][a] = __ffma2_rn(dup(wzy), s01[a], a01[c][b][a]);
          if (V4) a23[c][b][a] = __ffma2_rn(dup(wzy), s23[a], a23[c][b][a]);
          else a2[c][b][a] = fmaf(wzy, s23[a].x, a2[c][b][a]);
        }
      }
    }
  }
};

// the gather field on the 27 cells around one source cell, FP32 (x, y as a packed pair);
// cells beyond the block read the owning neighbour's active cell (the copy exchange of u*'s
// ghost cells folded into the load)
template <int D3>
struct GatherWindow {
  static constexpr int WK = D3 ? 3 : 1;
  float2 xy[WK][3][3];
  float z[WK][3][3];
  template <int GH>
  __device__ __forceinline__ void load(const Geo &G, const double *f, int m, int k, int jrow,
                                       int ci) {
#pragma unroll
    for (int c = 0; c < WK; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        // this cell's column of the (c, b) row; its x neighbours are the next words unless
        // the cell ends the block's row
        const int kk = D3 ? k - 1 + c : 0, jj = jrow - 1 + b;
        const long long rb = cell_at<GH>(G, m, 3, kk, jj, ci);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          long long at = (rb >= 0) ? rb + (a - 1) : -1;
          if ((a == 0 && ci == 0) || (a == 2 && ci == G.nx1 - 1)) at = cell_at<GH>(G, m, 3, kk, jj, ci - 1 + a);
          xy[c][b][a] = make_float2(0.0f, 0.0f);
          z[c][b][a] = 0.0f;
          if (at >= 0) {
            xy[c][b][a] = make_float2((float)f[at], (float)f[at + G.vstride]);
            z[c][b][a] = (float)f[at + 2 * G.vstride];
          }
        }
      }
  }
  // 3-D: the 27 cells from the gather window (cell + 1 in each direction: the stencil's
  // lowest cell, one below, is window index k, jrow, ci); consecutive threads read
  // consecutive cells, so every load of a warp is one coalesced 16-byte-per-lane access
  __device__ __forceinline__ void load4(const Geo &G, const float4 *W, int m, int k, int jrow,
                                        int ci) {
    const float4 *p = W + (((long long)m * G.W3 + k) * G.W2 + jrow) * G.W1 + ci;
#pragma unroll
    for (int c = 0; c < WK; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float4 v = __ldg(p + ((long long)c * G.W2 + b) * G.W1 + a);
          xy[c][b][a] = make_float2(v.x, v.y);
          z[c][b][a] = v.z;
        }
  }
  // 3-D, the window staged in shared memory (sw: the tile's rows plus one layer around them,
  // three planes, W1 cells per row); consecutive threads read consecutive 16-byte cells
  __device__ __forceinline__ void load4s(const float4 *sw, int W1, int rows, int cj, int ci) {
    const float4 *p = sw + cj * W1 + ci;
#pragma unroll
    for (int c = 0; c < WK; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const float4 v = p[(c * rows + b) * W1 + a];
          xy[c][b][a] = make_float2(v.x, v.y);
          z[c][b][a] = v.z;
        }
  }
  // u = sum over c of wz_c (sum over b of wy_b (sum over a of wx_a g_cba)): the three
  // directions one after the other, so the dependent chains are three FMAs long and the
  // planes' partial sums are independent of one another
  __device__ __forceinline__ void gather(const float wx[3], const float wy[3], const float wz[3],
                                         float2 &uxy, float &uz) const {
    float2 pxy[WK];
    float pz[WK];
#pragma unroll
    for (int c = 0; c < WK; ++c) {
      float2 sxy = make_float2(0.0f, 0.0f);
      float sz = 0.0f;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float2 txy = __fmul2_rn(dup(wx[0]), xy[c][b][0]);
        float tz = wx[0] * z[c][b][0];
#pragma unroll
        for (int a = 1; a < 3; ++a) {
          txy = __ffma2_rn(dup(wx[a]), xy[c][b][a], txy);
          tz = fmaf(wx[a], z[c][b][a], tz);
        }
        sxy = __ffma2_rn(dup(wy[b]), txy, sxy);
        sz = fmaf(wy[b], tz, sz);
      }
      pxy[c] = sxy;
      pz[c] = sz;
    }
    if (D3) {
      uxy = __fmul2_rn(dup(wz[0]), pxy[0]);
      uz = wz[0] * pz[0];
#pragma unroll
      for (int c = 1; c < WK; ++c) {
        uxy = __ffma2_rn(dup(wz[c]), pxy[c], uxy);
        uz = fmaf(wz[c], pz[c], uz);
      }
    } else {
      uxy = pxy[0];
      uz = pz[0];
    }
  }
};

// the sums of a source cell's particles of the pass (or of one slot, when the pass splits
// cells), staged in shared memory as float4 (values 0..3) at [(c*3 + b)*3 + a][cell or
// slot], for the window pass below
template <int MODE, int D3>
__device__ __forceinline__ void stage_sums(const CellSums<MODE, D3> &A, float4 *s_acc, int cl,
                                           int nct) {
  constexpr int WK = D3 ? 3 : 1;
#pragma unroll
  for (int c = 0; c < WK; ++c)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int a = 0; a < 3; ++a)
        s_acc[((c * 3 + b) * 3 + a) * nct + cl] =
            make_float4(A.val(c, b, a, 0), A.val(c, b, a, 1), A.val(c, b, a, 2),
                        FourValues<MODE>::value ? A.val(c, b, a, 3) : 0.0f);
}

// zero staged sums for a cell without particles in the pass
template <int D3>
__device__ __forceinline__ void stage_zero(float4 *s_acc, int cl, int nct) {
  constexpr int WK = D3 ? 3 : 1;
#pragma unroll
  for (int x = 0; x < WK * 9; ++x) s_acc[x * nct + cl] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// adds the tile's deposit window to the FP64 field, one add per window cell and value: a
// window cell (z plane c, row wy, column wx) sums the staged contributions of the up to 9
// source cells of its plane that reach it; window cells beyond the block go to the owning
// neighbour's active cell (the additive ghost exchange folded into the add)
// gs (the kick): this thread's FP64 sums of the values it adds (before the 1/V), the gas side
// of the tile's momentum ledger
template <int MODE, int D3, int GH>
__device__ __forceinline__ void add_window(const float4 *s_acc, const Geo &G, const TileArgs &T,
                                           int m, int k, int j0, int tj, const int *s_ss,
                                           double *gs) {
  constexpr int NC = FourValues<MODE>::value ? 4 : 3;
  constexpr int WK = D3 ? 3 : 1;
  const int nx1 = G.nx1, nct = tj * nx1;
  const int WI = nx1 + 2, WJ = tj + 2, nplane = WJ * WI;
  const double vinv = 1.0 / G.volm(m);             // (every deposited value is per unit volume)
  for (int t = threadIdx.x; t < WK * nplane; t += blockDim.x) {
    const int c = t / nplane, rem = t - c * nplane;
    const int wy = rem / WI, wx = rem - wy * WI;
    const long long at = cell_at<GH>(G, m, T.dnvar, D3 ? k - 1 + c : 0, j0 - 1 + wy, wx - 1);
    if (at < 0) continue;
    float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const int cj = wy - b;                       // source row reaching this row with offset b
      if (cj < 0 || cj >= tj) continue;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const int ci = wx - a;                     // source column reaching this column
        if (ci < 0 || ci >= nx1) continue;
        const int src = cj * nx1 + ci;
        if (!s_ss) {
          const float4 v = s_acc[((c * 3 + b) * 3 + a) * nct + src];
          s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
        } else {
          // (a pass with split cells: the sums are staged per slot, a cell's slots in a row)
          for (int q = s_ss[src]; q < s_ss[src + 1]; ++q) {
            const float4 v = s_acc[((c * 3 + b) * 3 + a) * nct + q];
            s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
          }
        }
      }
    }
    double *f = T.dfield + at;
    if (s.x != 0.0f) atomicAdd(f, (double)s.x * vinv);
    if (s.y != 0.0f) atomicAdd(f + G.vstride, (double)s.y * vinv);
    if (s.z != 0.0f) atomicAdd(f + 2 * G.vstride, (double)s.z * vinv);
    if (NC > 3 && s.w != 0.0f) atomicAdd(f + 3 * G.vstride, (double)s.w * vinv);
    if (MODE == MODE_KICK && gs) { gs[0] += (double)s.x; gs[1] += (double)s.y; gs[2] += (double)s.z; }
  }
}

// The window add of a 3-D tile in one pass whose threads are its cells (thread (cj, ci) holds
// cell (cj, ci)'s staged sums): thread (cj, ci) adds the window cells of its own column ci --
// target rows wy = cj + 1, and also row 0 (cj = 0) and row tj + 1 (cj = tj - 1) -- in the three
// planes, each the sum of the up to 9 staged contributions of source rows wy - b and columns
// ci + 1 - a; the threads of columns 0 and nx1 - 1 also add the halo columns x = -1 and x = nx1.
// Every thread has a fixed set of targets (no index division), a warp's loads of one
// contribution are consecutive in shared memory, and a target inside the block is indexed
// directly (cell_at only beyond the block's faces).  One FP64 add per window cell and value,
// as add_window.
template <int MODE, int GH>
__device__ __forceinline__ void add_window_cells(const float4 *s_acc, const Geo &G,
                                                 const TileArgs &T, int m, int k, int j0, int tj,
                                                 int cj, int ci, double *gs) {
  constexpr bool V4 = FourValues<MODE>::value;
  const int nx1 = G.nx1, nct = tj * nx1;
  const double vinv = 1.0 / G.volm(m);             // (every deposited value is per unit volume)
  auto put = [&](const float4 &v, int kt, int jt, int it) {
    long long at;
    if ((unsigned)kt < (unsigned)G.nx3 && (unsigned)jt < (unsigned)G.nx2 &&
        (unsigned)it < (unsigned)nx1)
      at = G.at(m, T.dnvar, 0, G.ks + kt, G.js + jt, G.is + it);
    else
      at = cell_at<GH>(G, m, T.dnvar, kt, jt, it);
    if (at < 0) return;
    double *f = T.dfield + at;
    if (v.x != 0.0f) atomicAdd(f, (double)v.x * vinv);
    if (v.y != 0.0f) atomicAdd(f + G.vstride, (double)v.y * vinv);
    if (v.z != 0.0f) atomicAdd(f + 2 * G.vstride, (double)v.z * vinv);
    if (V4 && v.w != 0.0f) atomicAdd(f + 3 * G.vstride, (double)v.w * vinv);
    if (MODE == MODE_KICK && gs) { gs[0] += (double)v.x; gs[1] += (double)v.y; gs[2] += (double)v.z; }
  };
  auto acc = [](float4 &s, const float4 &v) { s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w; };
  const int wy_lo = (cj == 0) ? 0 : cj + 1, wy_hi = (cj == tj - 1) ? tj + 1 : cj + 1;
  for (int wy = wy_lo; wy <= wy_hi; ++wy) {
    const int jt = j0 - 1 + wy;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float4 sm = make_float4(0.0f, 0.0f, 0.0f, 0.0f), sl = sm, sr = sm;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        const int sj = wy - b;
        if (sj < 0 || sj >= tj) continue;
        const float4 *row = s_acc + (size_t)((c * 3 + b) * 3) * nct + sj * nx1;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int si = ci + 1 - a;
          if (si >= 0 && si < nx1) acc(sm, row[(size_t)a * nct + si]);
        }
        if (ci == 0) acc(sl, row[ci]);                              // a = 0 -> x = -1
        if (ci == nx1 - 1) acc(sr, row[(size_t)2 * nct + ci]);      // a = 2 -> x = nx1
      }
      put(sm, k - 1 + c, jt, ci);
      if (ci == 0) put(sl, k - 1 + c, jt, -1);
      if (ci == nx1 - 1) put(sr, k - 1 + c, jt, nx1);
    }
  }
}

// dust_pc2_advance (src/dust/dust_push.cpp:132-245) of one particle in FP32 from u* gathered
// at its half-step gather position: the implicit midpoint velocity v_h (the 2x2 Coriolis solve
// and the vertical gravity of the shearing box), v <- 2 v_h - v0, the displacement dt xdot_h
// to the new position, and the drag impulse dt (u - v_h) / t_s handed to the gas.  With
// c = h/(t_s + h) (formed in FP64), 1/(1 + h/t_s) = 1 - c and (h/t_s)/(1 + h/t_s) = c, so the
// system (1 + l) v_h + K v_h = v0 + l u + G becomes v_h + (1 - c) K v_h = (1 - c)(v0 + G) + c u.
// The impulse is formed from the velocity change the particle received, less the Coriolis
// and gravity terms (the same quantity in exact arithmetic): dv = (v - v0) + 2 K v_h - 2 G.
__device__ __forceinline__ void pc2_particle(const Pc2Args &C, int three_d, float xh, float zh,
                                             const float v0[3], const float u[3], float c,
                                             bool shear_drift, float vn[3], float disp[3],
                                             float dv[3]) {
  const float s = 1.0f - c;
  float vh[3], kv[3] = {0.0f, 0.0f, 0.0f}, gv[3] = {0.0f, 0.0f, 0.0f};
  float r[3] = {s * v0[0] + c * u[0], s * v0[1] + c * u[1], s * v0[2] + c * u[2]};
  if (C.sbox && three_d) {
    if (C.strat) { gv[2] = -C.hom2 * zh; r[2] += s * gv[2]; }
    const float det = 1.0f + C.cxy * C.cyx * s * s;
    vh[0] = (r[0] + C.cxy * s * r[1]) / det;
    vh[1] = (r[1] - C.cyx * s * r[0]) / det;
    vh[2] = r[2];
    kv[0] = -C.cxy * vh[1]; kv[1] = C.cyx * vh[0];
  } else if (C.sbox) {
    // the 2-D (x, z) shearing box: the Coriolis pair is (x, z); const_accel_phi along z
    gv[2] = C.haphi; r[2] += s * gv[2];
    const float det = 1.0f + C.cxy * C.cyx * s * s;
    vh[0] = (r[0] + C.cxy * s * r[2]) / det;
    vh[2] = (r[2] - C.cyx * s * r[0]) / det;
    vh[1] = r[1];
    kv[0] = -C.cxy * vh[2]; kv[2] = C.cyx * vh[0];
  } else {
    vh[0] = r[0]; vh[1] = r[1]; vh[2] = r[2];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    vn[a] = 2.0f * vh[a] - v0[a];
    dv[a] = (vn[a] - v0[a]) + 2.0f * kv[a] - 2.0f * gv[a];
  }
  disp[0] = C.dt * vh[0];
  disp[1] = C.dt * (vh[1] - ((shear_drift && C.sbox && three_d) ? C.qom * xh : 0.0f));
  disp[2] = C.dt * vh[2];
}

// a CTA barrier entered by converged warps (the loops before it end at different iterations
// in different lanes; the barrier instruction assumes converged warps)
__device__ __forceinline__ void cta_sync(unsigned wmask) {
  __syncwarp(wmask);
  __syncthreads();
}

// the head of a tile's shared memory: the cell ranges, the slot starts of the pass (ints) and
// the centre mass of each cell (doubles, 8-byte aligned after the two int arrays), 16-byte
// aligned
__host__ __device__ inline size_t tile_head_bytes(int nct) {
  return (((size_t)(2 * nct + 2) * 4 + (size_t)nct * 8 + 15) & ~(size_t)15);
}

// shared memory of a tile: the head, then the larger of the pass rows and the staged sums
// (27 float4 per slot in 3-D, 9 in 2-D)
__host__ __device__ inline size_t tile_smem(int three_d, int tj, int nx1, int chunk) {
  const int nct = tj * nx1;
  const size_t rows = (size_t)kTileRows * chunk * 4;
  const size_t sums = (size_t)(three_d ? 27 : 9) * nct * 16;
  return tile_head_bytes(nct) + (rows > sums ? rows : sums);
}
// the staged window of a 3-D tile: its tj rows plus one row on each side, three planes, nx1 + 2
// cells of 16 bytes per row (after the rest, on a 128-byte boundary)
__host__ __device__ inline size_t tile_window_bytes(int tj, int nx1) {
  return (size_t)3 * (tj + 2) * (nx1 + 2) * 16;
}



// One CTA per tile of tj rows of one plane.  The tile's particles (one contiguous range of
// the sorted shadow) are cut into passes of at most chunk - 8, bulk-copied into shared
// memory.  In each pass every thread takes a slot: the particles of one source cell in the
// pass, or an even share of them when the pass covers fewer cells than there are threads
// (dense, clumped cells are split so that every thread has work).  A thread sums its slot's
// 27-point deposits in registers; the sums are staged in shared memory per slot and added
// to the field once per window cell and pass.  Operator, kick, pc2 predictor and advance:
// a gather phase (the 27 gather values of the slot's cell in registers) first writes each
// particle's deposit values (the kick: its velocity change; the advance: the gathered u*,
// which a coalesced per-particle step turns into the new state and the impulse) into its
// column, then the deposit phase sums them; the gather values and the sums are never live
// together.
// (at most 168 registers: three CTAs of 128 threads per SM)
template <int MODE, int D3, int SCHEME, int GH>
__global__ void __maxnreg__(168) k_tile(PBuf S, Geo G, TileArgs T,
                                        const __grid_constant__ CUtensorMap wmap) {
  // fields copied: ox oy oz cc m [vx vy vz] (the predictor: t_s in place of cc)
  constexpr int NF = (MODE == MODE_OP) ? 5 : 8;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_wsum[kMaxTileThreads / 32];
  __shared__ int s_wcnt[kMaxTileThreads / 32];
  __shared__ int s_split;                          // some cell of the pass has several slots
  __shared__ double s_ledger[6];                   // the kick tile's momentum ledger (FP64)
  const int nx1 = G.nx1, tj = T.tj;
  const int nct = tj * nx1;                        // source cells of the tile = threads
  const int CH = T.chunk;                          // buffer columns (multiple of 4)
  int *s_cs = (int *)smem;                         // [nct + 1] cell ranges
  int *s_ss = s_cs + (nct + 1);                    // [nct + 1] slot starts of the pass
  double *s_qt = (double *)(s_ss + (nct + 1));     // [nct] centre mass (Q/P), FP64
  float *s_f = (float *)(smem + tile_head_bytes(nct));   // [8][CH]
  float4 *s_acc = (float4 *)s_f;                   // the staged sums, after the rows
  // (GH bit 2, the gathering tiles of a 3-D mesh) the tile's gather window staged by a tensor
  // copy, after the rest on a 128-byte boundary
  constexpr bool kWin = D3 && MODE != MODE_QP && (GH & 4);
  float4 *s_win = (float4 *)(((uintptr_t)(smem + tile_smem(D3, tj, nx1, CH)) + 127) &
                             ~(uintptr_t)127);
  const int tid = threadIdx.x;
  const int lane = tid & 31, wid = tid >> 5;
  const unsigned wmask = (nct - (wid << 5)) >= 32 ? 0xffffffffu : ((1u << (nct - (wid << 5))) - 1u);
  const int nwarp = (nct + 31) >> 5;

  // the particle range [cb, ce) of a pass, field by field, rounded out to 16-byte groups; with
  // wz >= 0 (the first pass of a tile, kWin) also the tile's window: rows wj .. wj + tj + 1,
  // planes wz .. wz + 2 of the window tensor
  auto issue_pass = [&](int cb, int ce, int wj, int wz) {
    const int a0 = cb & ~3, a1 = (ce + 3) & ~3;
    const unsigned bytes = (unsigned)(a1 - a0) * 4u;
    const int fl[8] = {F_OX, F_OY, F_OZ, (MODE == MODE_PRED) ? F_TS : F_CC, F_M, F_VX, F_VY, F_VZ};
    const unsigned wbytes = (kWin && wz >= 0) ? (unsigned)tile_window_bytes(tj, nx1) : 0u;
    fence_proxy_async();
    mbar_arrive_tx(&bar, bytes * NF + wbytes);
#pragma unroll
    for (int f = 0; f < NF; ++f) bulk_copy(s_f + f * CH, S.f[fl[f]] + a0, bytes, &bar);
    if constexpr (kWin)
      if (wbytes) tensor_copy_4d(s_win, &wmap, 0, 0, wj, wz, &bar);
  };
  __shared__ int s_item;
  if (tid == 0) mbar_init(&bar, 1);
  unsigned parity = 0;                             // the copies' barrier phase, over all tiles
  // One tile per CTA (T.order null), or a persistent CTA taking tiles from the device work
  // queue -- T.order, heaviest first -- until the queue is empty.
  for (int item = 0;; ++item) {
    int t;
    if (!T.order) {
      if (item > 0) break;
      t = blockIdx.x;
    } else {
      if (tid == 0) s_item = atomicAdd(T.qhead, 1);
      cta_sync(wmask);
      const int q = s_item;
      if (q >= T.ntiles) break;
      t = T.order[q];
    }
    const int per_block = G.nx3 * T.tpp;
    const int m = t / per_block;
    t -= m * per_block;
    const int k = t / T.tpp;
    const int j0 = (t - k * T.tpp) * tj;
    const int c0 = encode(G, m, k, j0, 0);
    if (tid == 0) {
      // the first pass's copies go out before the cell ranges are read
      const int p0 = T.cstart[c0], p1 = T.cstart[c0 + nct];
      // (the failure-detection hook: the first tile of CTA 0 never issues its first copy, its
      // wait runs out)
      if (p1 > p0 && !(T.probe_timeout && blockIdx.x == 0 && item == 0))
        issue_pass(p0, min(p1, p0 + (CH - 8)), j0, kWin ? m * G.W3 + k : -1);
    }
    __syncwarp(wmask);
    for (int x = tid; x <= nct; x += blockDim.x) s_cs[x] = T.cstart[c0 + x];
    if (MODE == MODE_QP) s_qt[tid] = 0.0;
    for (int x = tid; x < 6; x += blockDim.x) s_ledger[x] = 0.0;   // (tiles of fewer threads)
    cta_sync(wmask);
    const int P0 = s_cs[0], P1 = s_cs[nct];
    const float inv_adt = (float)(1.0 / T.a_dt);
    const int CHP = CH - 8;                          // particles per pass (room to round out)
    const bool single = (P1 - P0) <= CHP;            // the whole tile in one pass

    for (int cb = P0; cb < P1; cb += CHP) {
      const int ce = min(P1, cb + CHP), cnt = ce - cb;
      const int a0 = cb & ~3, sh = cb - a0;
      if (tid == 0 && cb != P0) issue_pass(cb, ce, 0, -1);
      // (the warp reconverges before the barriers of the slot map: thread 0 must not arrive
      // at them apart from its warp)
      __syncwarp(wmask);
      // the slots of the pass: cell c gets q_c = ceil(n_c / R) of them, R the smallest share
      // with sum q_c <= threads (every cell one slot when the pass covers all the cells).  A
      // tile of one pass takes thread = cell directly (the uniform case)
      int cl = -1, lo = 0, hi = 0;
      if (single) {
        cl = tid; lo = s_cs[tid] - a0; hi = s_cs[tid + 1] - a0;
      } else {
        const int n_c = max(0, min(s_cs[tid + 1], ce) - max(s_cs[tid], cb));
        // (the cells with particles in the pass: per-warp ballots, summed after a barrier)
        const unsigned bal = __ballot_sync(wmask, n_c > 0);
        if (lane == 0) s_wcnt[wid] = __popc(bal);
        cta_sync(wmask);
        int ncp = 0;
        for (int w = 0; w < nwarp; ++w) ncp += s_wcnt[w];
        const int R = (ncp >= nct) ? cnt : (cnt + (nct - ncp) - 1) / (nct - ncp);
        const int q_c = (n_c > 0) ? (n_c + R - 1) / R : 0;
        int inc = q_c;                                 // block-wide inclusive scan of q_c
  #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(wmask, inc, o);
          if (lane >= o) inc += y;
        }
        if (lane == 31 || tid == nct - 1) s_wsum[wid] = inc;
        cta_sync(wmask);
        for (int w = 0; w < wid; ++w) inc += s_wsum[w];
        s_ss[tid + 1] = inc;
        if (tid == 0) s_ss[0] = 0;
        if (tid == nct - 1) s_split = inc > ncp;
        cta_sync(wmask);
        // this thread's slot: the last cell whose slots start at or before tid, an even share
        // of its particles in the pass (columns lo..hi of the rows)
        if (tid < s_ss[nct]) {
          int L = 0, H = nct - 1;
          while (L < H) {
            const int M = (L + H + 1) >> 1;
            if (s_ss[M] <= tid) L = M; else H = M - 1;
          }
          cl = L;
          const int qc = s_ss[cl + 1] - s_ss[cl], rk = tid - s_ss[cl];
          const int b0 = max(s_cs[cl], cb), len = min(s_cs[cl + 1], ce) - b0;
          lo = b0 + (len * rk) / qc - a0;
          hi = b0 + (len * (rk + 1)) / qc - a0;
        }
      }
      const int cj_l = (cl >= 0) ? cl / nx1 : 0, ci_l = (cl >= 0) ? cl - cj_l * nx1 : 0;
      const int jrow = j0 + cj_l;
      // the y offset of the weights: the particle's own, or (an imex stage with an implicit
      // shear shift) that of y + sh x, which the push kept inside the particle's cell
      auto oy_at = [&](int r) -> float {
        return (GH & 2) ? shifted_oy(G, T.shy, m, ci_l, s_f[r], s_f[CH + r]) : s_f[CH + r];
      };
      GatherWindow<D3> win;
      if constexpr (MODE != MODE_QP) {                 // (the loads fly with the copies)
        if constexpr (D3) {
          if constexpr (!kWin) win.load4(G, T.win4, m, k, jrow, ci_l);
        } else {
          win.template load<GH>(G, T.gfield, m, k, jrow, ci_l);
        }
      }
      const bool ok = mbar_wait(&bar, parity, T.err, wmask);
      parity ^= 1u;
      if (__syncthreads_or(!ok)) {
        // the copies never completed: wait once more (bounded) for them, then give up the tile
        mbar_wait(&bar, parity ^ 1u, T.err, wmask);
        return;
      }
      // (kWin: the staged window, complete with the first pass's copies)
      if constexpr (kWin) win.load4s(s_win, G.W1, tj + 2, cj_l, ci_l);
      if (MODE == MODE_QP) {
        CellSums<MODE, D3> qp;
        qp.zero();
        // (the centre mass m c summed in FP64 from the FP32 m and c the consistent kick uses:
        // exact products, so the dust share r q / qt of a cell sums to r q V over its particles)
        double qt = 0.0;
        for (int r = lo; r < hi; ++r) {
          float wx_[3], wy_[3], wz_[3];
          wts(SCHEME, s_f[r], wx_);
          wts(SCHEME, oy_at(r), wy_);
          if (D3) wts(SCHEME, s_f[2 * CH + r], wz_);
          const float mc = s_f[4 * CH + r] * s_f[3 * CH + r];
          qt += (double)s_f[4 * CH + r] * (double)s_f[3 * CH + r];
          qp.add(wx_, wy_, wz_, make_float2(mc, mc * s_f[5 * CH + r]),
                 make_float2(mc * s_f[6 * CH + r], mc * s_f[7 * CH + r]));
        }
        if (cl >= 0) atomicAdd(&s_qt[cl], qt);
        // the rows are read by now: their space takes the staged sums (per cell, or per slot
        // when the pass splits cells)
        cta_sync(wmask);
        const bool split = !single && s_split;
        if (!single && !split && s_ss[tid + 1] == s_ss[tid]) stage_zero<D3>(s_acc, tid, nct);
        if (cl >= 0) stage_sums<MODE, D3>(qp, s_acc, split ? tid : cl, nct);
        cta_sync(wmask);
        if (D3 && single) add_window_cells<MODE, GH>(s_acc, G, T, m, k, j0, tj, cj_l, ci_l, nullptr);
        else add_window<MODE, D3, GH>(s_acc, G, T, m, k, j0, tj, split ? s_ss : nullptr, nullptr);
      } else {
        // gather phase: the operator's m c u / V, the kick's velocity change, the predictor's
        // impulse and rate, or the advance's u*, into rows 5..7 (and 3)
        for (int r = lo; r < hi; ++r) {
          float wx_[3], wy_[3], wz_[3];
          wts(SCHEME, s_f[r], wx_);
          wts(SCHEME, oy_at(r), wy_);
          if (D3) wts(SCHEME, s_f[2 * CH + r], wz_);
          float2 uxy;
          float uz;
          win.gather(wx_, wy_, wz_, uxy, uz);
          const float c32 = s_f[3 * CH + r];
          if (MODE == MODE_OP) {
            const float mc = s_f[4 * CH + r] * c32;
            s_f[5 * CH + r] = mc * uxy.x; s_f[6 * CH + r] = mc * uxy.y; s_f[7 * CH + r] = mc * uz;
          } else if (MODE == MODE_PRED) {
            // dust_pc2_predictor (src/dust/dust_pm.cpp:141-193): rate m/(t_s V), impulse
            // -dt rate (u - v) from the old gas velocity m/rho of u1
            const float rate = s_f[4 * CH + r] / c32;
            const float vx = s_f[5 * CH + r], vy = s_f[6 * CH + r], vz = s_f[7 * CH + r];
            const float g = -T.pc.dt * rate;
            s_f[3 * CH + r] = rate;
            s_f[5 * CH + r] = g * (uxy.x - vx); s_f[6 * CH + r] = g * (uxy.y - vy);
            s_f[7 * CH + r] = g * (uz - vz);
          } else if (MODE == MODE_ADV) {
            s_f[5 * CH + r] = uxy.x; s_f[6 * CH + r] = uxy.y; s_f[7 * CH + r] = uz;
          } else {
            // GatherKickPMBR (src/dust/dust_pm.cpp:534-563): the applied velocity change
            const float vx = s_f[5 * CH + r], vy = s_f[6 * CH + r], vz = s_f[7 * CH + r];
            s_f[5 * CH + r] = (vx + c32 * (uxy.x - vx)) - vx;
            s_f[6 * CH + r] = (vy + c32 * (uxy.y - vy)) - vy;
            s_f[7 * CH + r] = (vz + c32 * (uz - vz)) - vz;
          }
        }
        // the kick's dust-side ledger of the pass, per thread: summed with the gas side of the
        // deposit phase in one warp sum (only their sum is used)
        double lk[3] = {0.0, 0.0, 0.0};
        if (MODE == MODE_KICK) {
          // the kicked velocities and rates of the pass, particle by particle (coalesced):
          // v <- v + dv, R <- dv / a_dt
          cta_sync(wmask);
          // (four particles per thread at a time, their velocity loads issued together)
          constexpr int U = 4;
          // the dust side of the tile's momentum ledger: the momentum m (v' - v) the particles
          // received (v' the stored FP32 velocity) and the part m (v' - v)/(a dt) - m R of the
          // rate that the FP32 rate R leaves out (the history term reads R).  v' - v is exact
          // in FP64 (two FP32 values), so each particle adds m (v' - v) and m R rounded once
          // in FP64; the rate part is formed from the thread's two sums at the end
          double le[3] = {0.0, 0.0, 0.0}, lm[3] = {0.0, 0.0, 0.0};
          for (int x0 = tid; x0 < cnt; x0 += U * blockDim.x) {
            float v[U][3];
  #pragma unroll
            for (int u = 0; u < U; ++u) {
              const int p = cb + min(x0 + u * (int)blockDim.x, cnt - 1);
              v[u][0] = S.f[F_VX][p]; v[u][1] = S.f[F_VY][p]; v[u][2] = S.f[F_VZ][p];
            }
  #pragma unroll
            for (int u = 0; u < U; ++u) {
              const int x = x0 + u * blockDim.x;
              if (x >= cnt) break;
              const int s = sh + x, p = cb + x;
              const float dv[3] = {s_f[5 * CH + s], s_f[6 * CH + s], s_f[7 * CH + s]};
              float vn[3], rn[3];
#pragma unroll
              for (int a = 0; a < 3; ++a) { vn[a] = v[u][a] + dv[a]; rn[a] = dv[a] * inv_adt; }
              S.f[F_VX][p] = vn[0]; S.f[F_VY][p] = vn[1]; S.f[F_VZ][p] = vn[2];
              S.f[F_RX][p] = rn[0]; S.f[F_RY][p] = rn[1]; S.f[F_RZ][p] = rn[2];
              if (T.ledger) {
                const double md = (double)s_f[4 * CH + s];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                  le[a] = fma(md, __dsub_rn((double)vn[a], (double)v[u][a]), le[a]);
                  if (T.hfield) lm[a] = fma(md, (double)rn[a], lm[a]);
                }
              }
            }
          }
          if (T.ledger) {
            const double iadt = 1.0 / T.a_dt;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              if (T.deposit) {
                lk[a] = le[a];
              } else {
                const double e = warp_sum(wmask, le[a]);
                if (lane == 0) atomicAdd(&s_ledger[a], e);
              }
              if (T.hfield) {
                // (sum of m (v' - v)/(a dt) - m R over the thread's particles)
                const double r = warp_sum(wmask, fma(le[a], iadt, -lm[a]));
                if (lane == 0) atomicAdd(&s_ledger[3 + a], r);
              }
            }
          }
        }
        if (MODE == MODE_ADV) {
          // the advanced particles of the pass, one per thread (coalesced): v, the
          // displacement to the new position (cells), the rate dv; their impulses -m dv / V
          // into rows 5..7
          cta_sync(wmask);
          for (int x = tid; x < cnt; x += blockDim.x) {
            const int s = sh + x, p = cb + x;
            const float v0[3] = {S.f[F_VX][p], S.f[F_VY][p], S.f[F_VZ][p]};
            const float u[3] = {s_f[5 * CH + s], s_f[6 * CH + s], s_f[7 * CH + s]};
            // (3-D shearing box: the half step left z_h in the z rate and the shear drift in
            // the displacement)
            const float zh = (T.pc.sbox && D3) ? S.f[F_RZ][p] : 0.0f;
            float vn[3], disp[3], dv[3];
            pc2_particle(T.pc, D3, 0.0f, zh, v0, u, s_f[3 * CH + s], false, vn, disp, dv);
            S.f[F_VX][p] = vn[0]; S.f[F_VY][p] = vn[1]; S.f[F_VZ][p] = vn[2];
            S.f[F_AX][p] += disp[0] * (float)G.inv_dx[0];
            S.f[F_AY][p] += disp[1] * (float)G.inv_dx[1];
            if (D3) S.f[F_AZ][p] += disp[2] * (float)G.inv_dx[2];
            S.f[F_RX][p] = dv[0]; S.f[F_RY][p] = dv[1]; S.f[F_RZ][p] = dv[2];
            const float f = -s_f[4 * CH + s];
            s_f[5 * CH + s] = f * dv[0]; s_f[6 * CH + s] = f * dv[1]; s_f[7 * CH + s] = f * dv[2];
          }
          cta_sync(wmask);
        }
        if (T.deposit) {
          // deposit phase: the sums of the values of this pass, added to the field
          CellSums<MODE, D3> sums;
          sums.zero();
          for (int r = lo; r < hi; ++r) {
            float wx_[3], wy_[3], wz_[3];
            wts(SCHEME, s_f[r], wx_);
            wts(SCHEME, oy_at(r), wy_);
            if (D3) wts(SCHEME, s_f[2 * CH + r], wz_);
            const float f = (MODE == MODE_KICK) ? -s_f[4 * CH + r] : 1.0f;
            sums.add(wx_, wy_, wz_, make_float2(f * s_f[5 * CH + r], f * s_f[6 * CH + r]),
                     make_float2(f * s_f[7 * CH + r], (MODE == MODE_PRED) ? s_f[3 * CH + r] : 0.0f));
          }
          // the rows are read by now: their space takes the staged sums (per cell, or per slot
          // when the pass splits cells)
          cta_sync(wmask);
          const bool split = !single && s_split;
          if (!single && !split && s_ss[tid + 1] == s_ss[tid]) stage_zero<D3>(s_acc, tid, nct);
          if (cl >= 0) stage_sums<MODE, D3>(sums, s_acc, split ? tid : cl, nct);
          cta_sync(wmask);
          double gs[3] = {0.0, 0.0, 0.0};
          if (D3 && single) add_window_cells<MODE, GH>(s_acc, G, T, m, k, j0, tj, cj_l, ci_l, gs);
          else add_window<MODE, D3, GH>(s_acc, G, T, m, k, j0, tj, split ? s_ss : nullptr, gs);
          if (MODE == MODE_KICK && T.ledger) {
            // the gas side of the tile's ledger: what this pass added, with the dust side,
            // summed over the CTA
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              const double w = warp_sum(wmask, gs[a] + lk[a]);
              if (lane == 0) atomicAdd(&s_ledger[a], w);
            }
          }
        }
      }
      // the next pass's copies overwrite the rows (and its slots the slot starts)
      cta_sync(wmask);
    }
    if (MODE == MODE_KICK && T.ledger && P1 > P0) {
      // the tile's momentum ledger closed: what the gas received from the FP32 sums and what
      // the particles received differ by the FP32 rounding of weights, products and sums; the
      // difference goes to the gas in equal parts at the first cell of each warp's cells, so
      // that gas and dust exchange exactly opposite momenta (FP64 round-off) and no cell takes
      // a tile's worth of rounding.  The rate's rounding goes to the history field the same
      // way (the next stage's history term adds it to the gas as it adds the gas rate)
      cta_sync(wmask);
      if (lane == 0) {
        const double share = 1.0 / (G.volm(m) * (double)nwarp);
        const int cj = tid / nx1, ci = tid - cj * nx1;
        const long long at = G.at(m, 3, 0, G.ks + k, G.js + j0 + cj, G.is + ci);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double r = -s_ledger[a];
          if (r != 0.0) atomicAdd(&T.dfield[at + a * G.vstride], r * share);
          if (T.hfield && s_ledger[3 + a] != 0.0)
            atomicAdd(&T.hfield[at + a * G.vstride], s_ledger[3 + a] * share);
        }
      }
    }
    if (MODE == MODE_QP) {
      // centre mass m c / V of the cell (dust_imex_point_center_mass): only this cell's
      // particles have it as their centre, so it is stored, not added
      const int cj = tid / nx1, ci = tid - cj * nx1;
      T.res[G.at(m, 4, 3, G.ks + k, G.js + j0 + cj, G.is + ci)] = s_qt[tid] / G.volm(m);
    }
    // (every thread is done with this tile's shared memory before the next tile's copies)
    cta_sync(wmask);
  }
}

// The device work queue of a stage: every tile of the mesh ordered by its particle count,
// heaviest first (buckets of equal log2 count, in descending order; a tile's place inside its
// bucket does not matter), so that the persistent tile launches start the long tiles first
// and finish on short ones.  One CTA; also clears the stage's queue counters.
__global__ void __launch_bounds__(1024) k_tile_order(const int *cstart, Geo G, int tj, int tpp,
                                                     int ntiles, int *order, int *qhead) {
  __shared__ int hist[33], base[33];
  const int nct = tj * G.nx1, per_block = G.nx3 * tpp;
  auto bucket = [&](int t) {
    const int m = t / per_block, r = t - m * per_block, k = r / tpp, j0 = (r - k * tpp) * tj;
    const int c0 = encode(G, m, k, j0, 0);
    const int cost = cstart[c0 + nct] - cstart[c0];
    return cost > 0 ? __clz(cost) : 32;           // 32 - log2 size: heavy tiles first
  };
  for (int b = threadIdx.x; b < 33; b += blockDim.x) hist[b] = 0;
  if (threadIdx.x < kQueues) qhead[threadIdx.x] = 0;
  __syncthreads();
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) atomicAdd(&hist[bucket(t)], 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int b = 0; b < 33; ++b) { base[b] = run; run += hist[b]; }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ntiles; t += blockDim.x) order[atomicAdd(&base[bucket(t)], 1)] = t;
}

// m/rho of a gas field on every cell, ghosts included: the predictor's gather field
__global__ void k_gas_velocity(const double *u, int nv, double *out, long long per,
                               long long total) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const long long m = idx / per, c = idx - m * per;
  const double inv = 1.0 / u[(m * nv) * per + c];
  for (int v = 0; v < 3; ++v) out[(m * 3 + v) * per + c] = u[(m * nv + 1 + v) * per + c] * inv;
}

// The pc2 advance of the edge bin: particles whose gather position lies beyond a physical x3
// face or a shear-periodic x1 face of their block.  There the gather and the deposit use the
// block's own ghost cells (u* beyond the face as the FP64 form has it; the deposit's ghost
// exchange folds, drops or remaps it), as dust_pc2_advance does for every particle.  One
// thread per particle, the same FP32 arithmetic as the advance tiles, FP64 atomics.  The
// shadow keeps such a particle at its old position, so its displacement is the whole step.
template <int SCHEME>
__global__ void __launch_bounds__(kT) k_pc2_edge(PBuf S, Geo G, TileArgs T) {
  const int e0 = T.cstart[G.ncell], e1 = T.cstart[G.ncell + 1];
  const double vinv = 1.0 / G.vol;
  const int nax = G.three_d ? 3 : 2;
  for (int p = e0 + blockIdx.x * blockDim.x + threadIdx.x; p < e1; p += gridDim.x * blockDim.x) {
    int m, k, j, i;
    decode(G, S.cell[p], m, k, j, i);
    const double *sz = G.mb + (long long)m * 9;
    const float v0[3] = {S.f[F_VX][p], S.f[F_VY][p], S.f[F_VZ][p]};
    const float o[3] = {S.f[F_OX][p], S.f[F_OY][p], S.f[F_OZ][p]};
    // the gather position in block-local cells, as the half-step push forms it
    float xsh = 0.0f;
    if (T.pc.sbox && G.three_d)
      xsh = T.pc.qom * (float)(sz[X1MIN] + ((double)i + (double)o[0]) * G.dx[0]);
    const float xdot[3] = {v0[0], v0[1] - xsh, v0[2]};
    const int idx[3] = {i, j, k}, nx[3] = {G.nx1, G.nx2, G.nx3};
    float g[3], w[3][3];
    int ig[3];
    bool in = true;
    for (int a = 0; a < 3; ++a) {
      g[a] = (float)idx[a] + o[a];
      if (a < nax) g[a] += T.pc.hdx[a] * xdot[a];
      if (a == 1 && T.pc.gy != 0.0f) g[1] += T.pc.gy * (float)(sz[X1MIN] + (double)g[0] * G.dx[0]);
      ig[a] = (a < nax) ? (int)floorf(g[a]) : idx[a];
      wts(SCHEME, (a < nax) ? g[a] - (float)ig[a] : 0.5f, w[a]);
      if (a < nax && (ig[a] < -1 || ig[a] > nx[a])) in = false;
    }
    if (!in) { report(T.err, DUSTB_ERR_HALO); continue; }
    // the gather from the block's own cells, ghost cells included
    const int clo = G.three_d ? 0 : 1, chi = G.three_d ? 2 : 1;
    float u[3] = {0.0f, 0.0f, 0.0f};
    for (int c = clo; c <= chi; ++c)
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
          const float wt = (G.three_d ? w[2][c] : 1.0f) * w[1][b] * w[0][a];
          const long long at = G.at(m, 3, 0, G.three_d ? G.ks + ig[2] - 1 + c : G.ks,
                                    G.js + ig[1] - 1 + b, G.is + ig[0] - 1 + a);
          u[0] += wt * (float)T.gfield[at];
          u[1] += wt * (float)T.gfield[at + G.vstride];
          u[2] += wt * (float)T.gfield[at + 2 * G.vstride];
        }
    const float xh = (float)(sz[X1MIN] + (double)g[0] * G.dx[0]);
    const float zh = G.three_d ? (float)(sz[X3MIN] + (double)g[2] * G.dx[2]) : 0.0f;
    float vn[3], disp[3], dv[3];
    pc2_particle(T.pc, G.three_d, xh, zh, v0, u, S.f[F_CC][p], true, vn, disp, dv);
    S.f[F_VX][p] = vn[0]; S.f[F_VY][p] = vn[1]; S.f[F_VZ][p] = vn[2];
    S.f[F_AX][p] += disp[0] * (float)G.inv_dx[0];
    S.f[F_AY][p] += disp[1] * (float)G.inv_dx[1];
    if (G.three_d) S.f[F_AZ][p] += disp[2] * (float)G.inv_dx[2];
    S.f[F_RX][p] = dv[0]; S.f[F_RY][p] = dv[1]; S.f[F_RZ][p] = dv[2];
    if (!T.deposit) continue;
    const float f = -S.f[F_M][p];
    for (int c = clo; c <= chi; ++c)
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
          const float wt = f * (G.three_d ? w[2][c] : 1.0f) * w[1][b] * w[0][a];
          if (wt == 0.0f) continue;
          const long long at = G.at(m, 3, 0, G.three_d ? G.ks + ig[2] - 1 + c : G.ks,
                                    G.js + ig[1] - 1 + b, G.is + ig[0] - 1 + a);
          atomicAdd(&T.dfield[at], (double)(wt * dv[0]) * vinv);
          atomicAdd(&T.dfield[at + G.vstride], (double)(wt * dv[1]) * vinv);
          atomicAdd(&T.dfield[at + 2 * G.vstride], (double)(wt * dv[2]) * vinv);
        }
  }
}

// The imex stage's edge bin under an implicit shear shift: particles whose weight position
// y + sh x lies in a cell next to their own.  One thread per particle with the tiles' FP32
// arithmetic at the shifted position and FP64 atomics: Q/P with the centre mass into the
// particle's own cell (after the Q/P tiles stored theirs), the dc1 operator, the
// gather-kick-deposit.  3-D.
template <int MODE, int SCHEME, int GH>
__global__ void __launch_bounds__(kT) k_shift_edge(PBuf S, Geo G, TileArgs T) {
  const int e0 = T.cstart[G.ncell], e1 = T.cstart[G.ncell + 1];
  const double vinv = 1.0 / G.vol;
  const float inv_adt = (float)(1.0 / T.a_dt);
  for (int p = e0 + blockIdx.x * blockDim.x + threadIdx.x; p < e1; p += gridDim.x * blockDim.x) {
    int m, k, j, i;
    decode(G, S.cell[p], m, k, j, i);
    const float ox = S.f[F_OX][p];
    float oy = shifted_oy(G, T.shy, m, i, ox, S.f[F_OY][p]);
    const float fl = floorf(oy);
    const int jc = j + (int)fl;                   // the cell of the shifted position
    oy = __fsub_rn(oy, fl);
    if (oy >= 1.0f) oy = 0.99999994f;
    float wx[3], wy[3], wz[3];
    wts(SCHEME, ox, wx); wts(SCHEME, oy, wy); wts(SCHEME, S.f[F_OZ][p], wz);
    const float cc = S.f[F_CC][p], mass = S.f[F_M][p];
    const float mc = mass * cc;
    if (MODE == MODE_QP) {
      const float v[3] = {S.f[F_VX][p], S.f[F_VY][p], S.f[F_VZ][p]};
      for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 3; ++b)
          for (int a = 0; a < 3; ++a) {
            const float w = wz[c] * wy[b] * wx[a] * mc;
            if (w == 0.0f) continue;
            const long long at = cell_at<GH>(G, m, T.dnvar, k - 1 + c, jc - 1 + b, i - 1 + a);
            if (at < 0) continue;
            atomicAdd(&T.dfield[at], (double)w * vinv);
            atomicAdd(&T.dfield[at + G.vstride], (double)(w * v[0]) * vinv);
            atomicAdd(&T.dfield[at + 2 * G.vstride], (double)(w * v[1]) * vinv);
            atomicAdd(&T.dfield[at + 3 * G.vstride], (double)(w * v[2]) * vinv);
          }
      atomicAdd(&T.res[G.at(m, 4, 3, G.ks + k, G.js + j, G.is + i)], (double)mc * vinv);
      continue;
    }
    float u[3] = {0.0f, 0.0f, 0.0f};
    for (int c = 0; c < 3; ++c)
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
          const float w = wz[c] * wy[b] * wx[a];
          const long long at = cell_at<GH>(G, m, 3, k - 1 + c, jc - 1 + b, i - 1 + a);
          if (at < 0) continue;
          u[0] += w * (float)T.gfield[at];
          u[1] += w * (float)T.gfield[at + G.vstride];
          u[2] += w * (float)T.gfield[at + 2 * G.vstride];
        }
    float val[3];
    if (MODE == MODE_OP) {
      for (int q = 0; q < 3; ++q) val[q] = mc * u[q];
    } else {
      // GatherKickPMBR (src/dust/dust_pm.cpp:534-563): the applied velocity change
      const float v0[3] = {S.f[F_VX][p], S.f[F_VY][p], S.f[F_VZ][p]};
      for (int q = 0; q < 3; ++q) val[q] = (v0[q] + cc * (u[q] - v0[q])) - v0[q];
      S.f[F_VX][p] = v0[0] + val[0]; S.f[F_VY][p] = v0[1] + val[1]; S.f[F_VZ][p] = v0[2] + val[2];
      S.f[F_RX][p] = val[0] * inv_adt; S.f[F_RY][p] = val[1] * inv_adt; S.f[F_RZ][p] = val[2] * inv_adt;
      if (!T.deposit) continue;
      const float f = -mass;
      for (int q = 0; q < 3; ++q) val[q] *= f;
    }
    for (int c = 0; c < 3; ++c)
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
          const float w = wz[c] * wy[b] * wx[a];
          if (w == 0.0f) continue;
          const long long at = cell_at<GH>(G, m, 3, k - 1 + c, jc - 1 + b, i - 1 + a);
          if (at < 0) continue;
          for (int q = 0; q < 3; ++q) atomicAdd(&T.dfield[at + q * G.vstride], (double)(w * val[q]) * vinv);
        }
  }
}

// ---- kernel timing ------------------------------------------------------------------------
struct Timing {
  bool on = false;
  std::vector<cudaEvent_t> ev[DUSTB_K_NKERNELS];   // start, stop pairs
  size_t used[DUSTB_K_NKERNELS] = {0};
};
Timing g_timing;

struct Scope {
  int id; cudaStream_t st; bool on;
  Scope(int id_, cudaStream_t s) : id(id_), st(s), on(g_timing.on) {
    if (!on) return;
    auto &v = g_timing.ev[id];
    size_t u = g_timing.used[id];
    while (v.size() < u + 2) { cudaEvent_t e; cudaEventCreate(&e); v.push_back(e); }
    cudaEventRecord(v[u], st);
  }
  ~Scope() {
    if (!on) return;
    size_t &u = g_timing.used[id];
    cudaEventRecord(g_timing.ev[id][u + 1], st);
    u += 2;
  }
};

struct Cfg {
  int tj, chunk, tpp;
  int probe_timeout;
  int grid;                      // 1: one CTA per tile; 0: persistent CTAs on the work queue
  int wtma;                      // 3-D: the gathering tiles stage their window by a tensor copy
};

// the default particles per pass: the largest multiple of 4 that lets as many CTAs share an
// SM as their registers allow (about 168 per thread), so that a typical tile's particles
// fit one pass (a second pass costs a second window flush)
// (extra: shared memory a CTA needs beyond the head and the rows: the staged window)
int default_chunk(int tj, int nx1, long long extra = 0) {
  const int nct = tj * nx1;
  int ctas = 65536 / (168 * nct);
  ctas = ctas < 1 ? 1 : (ctas > 8 ? 8 : ctas);
  const long long per = 233472 / ctas - 2560 - 64;     // less a reserve and the statics
  long long ch = (per - (long long)tile_head_bytes(nct) - extra) / (kTileRows * 4);
  ch &= ~3LL;
  return (int)(ch < 64 ? 64 : (ch > 8192 ? 8192 : ch));
}

bool pick_cfg(const dustb_mesh &ms, const dustb_mixed_params *mp, Cfg &cf) {
  const int nx1 = ms.nx1, nx2 = ms.multi_d ? ms.nx2 : 1;
  const int base = mp->variant & ~(DUSTB_MIXED_GRID_TILES | DUSTB_MIXED_NO_LEDGER |
                                   DUSTB_MIXED_WINDOW_TMA);
  if ((base != 0 && base != DUSTB_MIXED_PROBE_COPY_TIMEOUT) || nx1 > kMaxTileThreads)
    return false;
  cf.grid = (mp->variant & DUSTB_MIXED_GRID_TILES) ? 1 : 0;
  // (a box row of the window tensor holds at most 256 cells)
  cf.wtma = ((mp->variant & DUSTB_MIXED_WINDOW_TMA) && ms.three_d && nx1 + 2 <= 256) ? 1 : 0;
  int tj = mp->rows_per_tile;
  if (tj <= 0) {
    tj = 1;
    for (int t = nx2; t >= 1; --t)
      if (nx2 % t == 0 && t * nx1 <= 128) { tj = t; break; }
  }
  if (nx2 % tj != 0 || tj * nx1 > kMaxTileThreads) return false;
  cf.tj = tj;
  cf.chunk = mp->chunk > 0 ? mp->chunk
                           : default_chunk(tj, nx1, cf.wtma ? 128 + (long long)tile_window_bytes(tj, nx1) : 0);
  if (cf.chunk < 64 || cf.chunk > 8192 || (cf.chunk & 3)) return false;
  cf.tpp = nx2 / tj;
  cf.probe_timeout = (base == DUSTB_MIXED_PROBE_COPY_TIMEOUT);
  // every tile form must fit the 227 KiB of shared memory a CTA can have (less the barrier)
  const size_t extra = cf.wtma ? 128 + tile_window_bytes(tj, nx1) : 0;
  if (tile_smem(ms.three_d, tj, nx1, cf.chunk) + extra > 227 * 1024 - 256) return false;
  return true;
}

// the tensor map of the gather window (float4 cells, W1 x W2 x W3 per block): 4-D as (the four
// floats of a cell, x, y, z over all blocks), a box of one tile's window (all W1 cells of tj + 2
// rows in 3 planes); false when the driver's encoder is not available or refuses the map
bool window_map(const Geo &G, const float4 *win, int tj, CUtensorMap &map) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  if (!win || ((uintptr_t)win & 15) || G.W1 > 256 || tj + 2 > 256) return false;
  const cuuint64_t dims[4] = {4, (cuuint64_t)G.W1, (cuuint64_t)G.W2,
                              (cuuint64_t)G.W3 * (cuuint64_t)G.nmb};
  const cuuint64_t strides[3] = {16, 16ull * G.W1, 16ull * G.W1 * G.W2};
  const cuuint32_t box[4] = {4, (cuuint32_t)G.W1, (cuuint32_t)(tj + 2), 3};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)win, dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// GH bit 2: the form that stages the window (wm its tensor map), chosen here when the
// configuration asks for it and the map can be made
template <int MODE, int D3, int SCHEME, int GH>
int launch_tile_d(const Geo &G, const Cfg &cf, const PBuf &cur, const TileArgs &T, cudaStream_t st,
                  const CUtensorMap *wm = nullptr) {
  if constexpr (D3 && MODE != MODE_QP && !(GH & 4)) {
    if (cf.wtma) {
      CUtensorMap m4;
      if (window_map(G, T.win4, cf.tj, m4))
        return launch_tile_d<MODE, D3, SCHEME, GH | 4>(G, cf, cur, T, st, &m4);
    }
  }
  CUtensorMap wmap;
  std::memset(&wmap, 0, sizeof(wmap));
  if (wm) wmap = *wm;
  const long long tiles = (long long)G.nmb * G.nx3 * cf.tpp;
  const size_t sm = tile_smem(D3, cf.tj, G.nx1, cf.chunk) +
                    ((GH & 4) ? 128 + tile_window_bytes(cf.tj, G.nx1) : 0);
  const int threads = cf.tj * G.nx1;
  static size_t configured = 0;
  // the CTAs of this kernel one SM holds at this shared-memory size and block (for the
  // persistent launch), looked up once per size
  static size_t occ_sm = 0;
  static int occ_threads = 0, occ = 0, nsm = 0;
  if (sm > 48 * 1024 && sm > configured) {
    cudaFuncSetAttribute(k_tile<MODE, D3, SCHEME, GH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    configured = sm;
  }
  long long grid = tiles;
  if (T.order) {
    if (occ_sm != sm || occ_threads != threads || nsm == 0) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile<MODE, D3, SCHEME, GH>, threads, sm);
      occ_sm = sm; occ_threads = threads;
    }
    const long long resident = (long long)(occ > 0 ? occ : 1) * (nsm > 0 ? nsm : 1);
    grid = tiles < resident ? tiles : resident;
  }
  k_tile<MODE, D3, SCHEME, GH><<<(unsigned)grid, threads, sm, st>>>(cur, G, T, wmap);
  return dustb_host::launch_status("mixed tile");
}

// the stage's work queue (the tiles of the sorted copy heaviest first) unless the
// configuration asks for one CTA per tile
int build_queue(const MState &S, const Geo &G, const Cfg &cf, TileArgs &T, cudaStream_t st) {
  T.order = nullptr; T.qhead = nullptr;
  if (cf.grid) return DUSTB_OK;
  T.ntiles = G.nmb * G.nx3 * cf.tpp;
  k_tile_order<<<1, 1024, 0, st>>>(S.cstart, G, cf.tj, cf.tpp, T.ntiles, S.tile_order, S.qhead);
  T.order = S.tile_order;
  T.qhead = S.qhead;
  return dustb_host::launch_status("mixed tile queue");
}

// the kernel of one dimensionality, ghost mode (GH bit 0) and implicit-shift form (bit 1)
template <int MODE, int D3, int GH>
int launch_tile_s(const Geo &G, const Cfg &cf, const PBuf &cur, const TileArgs &T, cudaStream_t st) {
  if (G.scheme == 2) return launch_tile_d<MODE, D3, 2, GH>(G, cf, cur, T, st);
  if (G.scheme == 1) return launch_tile_d<MODE, D3, 1, GH>(G, cf, cur, T, st);
  return launch_tile_d<MODE, D3, 0, GH>(G, cf, cur, T, st);
}

template <int MODE>
int launch_tile(const MState &S, const PBuf &cur, const Geo &G, const Cfg &cf, TileArgs T,
                cudaStream_t st, int qslot) {
  T.tj = cf.tj; T.chunk = cf.chunk; T.tpp = cf.tpp; T.cstart = S.cstart;
  if (T.qhead) T.qhead = S.qhead + qslot;
  T.probe_timeout = cf.probe_timeout;
  // one kernel per dimensionality and deposit scheme (no per-particle scheme selection); the
  // weights shifted by an imex stage's implicit shear shift only in the kernels of that form
  constexpr bool kImex = MODE == MODE_QP || MODE == MODE_OP || MODE == MODE_KICK;
  if constexpr (kImex) {
    if (T.shy != 0.0f) {
      if (!G.three_d) return launch_tile_s<MODE, 0, 2>(G, cf, cur, T, st);
      return G.ghost ? launch_tile_s<MODE, 1, 3>(G, cf, cur, T, st)
                     : launch_tile_s<MODE, 1, 2>(G, cf, cur, T, st);
    }
  }
  // (ghost mode: physical x3 or shear-periodic x1 faces, 3-D only)
  if (!G.three_d) return launch_tile_s<MODE, 0, 0>(G, cf, cur, T, st);
  return G.ghost ? launch_tile_s<MODE, 1, 1>(G, cf, cur, T, st)
                 : launch_tile_s<MODE, 1, 0>(G, cf, cur, T, st);
}

// the edge bin of an imex stage with an implicit shear shift (after the mode's tiles)
template <int MODE>
int launch_shift_edge(const MState &S, const PBuf &cur, const Geo &G, TileArgs T, cudaStream_t st) {
  T.cstart = S.cstart;
  const unsigned nb = 148 * 4;
#define DUSTB_SE(SC, GHF) k_shift_edge<MODE, SC, GHF><<<nb, kT, 0, st>>>(cur, G, T)
  if (G.ghost) {
    if (G.scheme == 2) DUSTB_SE(2, 1); else if (G.scheme == 1) DUSTB_SE(1, 1); else DUSTB_SE(0, 1);
  } else {
    if (G.scheme == 2) DUSTB_SE(2, 0); else if (G.scheme == 1) DUSTB_SE(1, 0); else DUSTB_SE(0, 0);
  }
#undef DUSTB_SE
  return dustb_host::launch_status("mixed shear-shift edge");
}

// the gather window of a 3-D mesh from the FP64 gather field f (after its ghost exchange in
// ghost mode); nothing in 2-D
int gather_window(const MState &S, const Geo &G, const dustb_mesh &ms, const double *f,
                  TileArgs &T, cudaStream_t st) {
  T.win4 = S.win;
  if (!ms.three_d) return DUSTB_OK;
  Scope sc(DUSTB_K_WINDOW, st);
  const long long n = nwin(ms);
  const unsigned nb = (unsigned)((n + 255) / 256 < 148LL * 16 ? (n + 255) / 256 : 148LL * 16);
  if (G.ghost) k_gather_window<1><<<nb, 256, 0, st>>>(f, S.win, G);
  else k_gather_window<0><<<nb, 256, 0, st>>>(f, S.win, G);
  return dustb_host::launch_status("mixed gather window");
}

// sort copy src into dst by the cells it holds (histogram, scan, moves)
int sort_into(const MState &S, const PBuf &src, const PBuf &dst, const dustb_mesh &ms, int n,
              cudaStream_t st) {
  const long long ncell = ncell_of(ms);
  cudaMemsetAsync(S.cstart, 0, 4 * (size_t)nbins(ncell), st);
  if (n > 0) k_hist<<<nblk(n), kT, 0, st>>>(src.cell, n, S.cstart);
  int rc = exclusive_scan(S.cstart, nbins(ncell), S.bsum, st);
  if (rc) return rc;
  cudaMemcpyAsync(S.cursor, S.cstart, 4 * (size_t)nbins(ncell), cudaMemcpyDeviceToDevice, st);
  if (n > 0) k_sortmove<<<nblk(n), kT, 0, st>>>(src, dst, n, S.cursor);
  return dustb_host::launch_status("mixed sort");
}

// import and export read and write the reference rows: they must be attached
bool rows_attached(const dustb_ctx *c) {
  return c->part.npart == 0 || (c->part.pr && c->part.pi);
}

bool params_ok(const dustb_ctx *c, const dustb_mixed_params *mp) {
  if (!dustb_cells::ctx_valid(c) || !mp) return false;
  if (c->mesh.nghbr_ml) {
    // a refined mesh: periodic, 3-D, with its deposit remap and copy-exchange scratch
    const dustb_mesh &ms = c->mesh;
    if (!ms.mb_lev || !ms.three_d || ms.x3bc != DUSTB_X3_PERIODIC || ms.shear_x1) return false;
    if (!mp->plan || !mp->coarse || mp->root_level < 0) return false;
  }
  for (int a = 0; a < 3; ++a)
    if (!(mp->dx[a] > 0.0)) return false;
  if (ncell_of(c->mesh) >= (1LL << 31) - 2) return false;   // (cells and the edge bin)
  return true;
}


// the geometry's tables and outputs are there
bool geo_ok(const dustb_mixed_params *mp, const Geo &G) {
  if (G.sb_on && (!G.sb_gid || G.sb_nb2 <= 0 || G.sb_nb3 <= 0)) return false;
  if (G.x3bc == DUSTB_X3_OUTFLOW && !mp->x3_removed) return false;
  return true;
}

// ghost mode: the FP64 exchanges around the tiles (additive: x3 fold or drop and the shear
// remap included; copy: the shear remap and the x3 boundary values of u*)
// (a refined mesh: the general deposit remap and the multilevel copy exchange)
int ghost_add_if(const dustb_ctx *c, const Geo &G, double *f, int nvar, cudaStream_t st,
                 const dustb_mixed_params *mp) {
  if (G.ml) return dustb_ghost_add_plan(c, mp->plan, f, nvar, st);
  return G.ghost ? dustb_ghost_add(c, f, nvar, st) : DUSTB_OK;
}
int ghost_copy_if(const dustb_ctx *c, const Geo &G, double *f, cudaStream_t st,
                  const dustb_mixed_params *mp) {
  if (G.ml) return dustb_ghost_copy_ml(c, f, 3, mp->coarse, mp->coarse_bytes, st);
  return G.ghost ? dustb_ghost_copy(c, f, 3, 1, st) : DUSTB_OK;
}

// the pc2 constants of a cycle (dust_push.cpp:132-245), rounded once to FP32
Pc2Args make_pc2(const dustb_ctx *c, const Geo &G, double dt) {
  Pc2Args a{};
  const double h = 0.5 * dt, om = c->phys.omega0, q = c->phys.qshear;
  a.dt = (float)dt; a.h = (float)h;
  a.cxy = (float)(2.0 * h * om); a.cyx = (float)(h * (2.0 - q) * om);
  a.qom = (float)(q * om); a.hom2 = (float)(h * om * om);
  a.haphi = (float)(h * c->phys.const_accel_phi);
  for (int x = 0; x < 3; ++x) a.hdx[x] = (float)(h * G.inv_dx[x]);
  a.sbox = c->phys.shearing_box; a.strat = c->phys.stratified;
  a.gy = (a.sbox && G.three_d) ? (float)(q * om * h * G.inv_dx[1]) : 0.0f;
  return a;
}

// one push: count (the new cells and their histogram), the scan of the bins, the moves
int push_sort(const MState &S, const PBuf &src, const PBuf &dst, const Geo &G, int n,
              long long ncell, const PushArgs &P, cudaStream_t st) {
  int rc;
  {
    Scope sc(DUSTB_K_COUNT, st);
    cudaMemsetAsync(S.cstart, 0, 4 * (size_t)nbins(ncell), st);
    if (n > 0) {
#define DUSTB_COUNT(K, SPF) k_count<K, SPF><<<nblk(n), kT, 0, st>>>(src, S.key, S.cstart, G, n, P)
      // (physical x3 or shear faces; a refined mesh carries its crossings in the periodic form)
      if (G.ml) {
        if (P.kind == PK_HALF) DUSTB_COUNT(PK_HALF, 2);
        else if (P.kind == PK_FULL) DUSTB_COUNT(PK_FULL, 2);
        else DUSTB_COUNT(PK_IMEX, 2);
      } else if (G.ghost) {
        if (P.kind == PK_HALF) DUSTB_COUNT(PK_HALF, 1);
        else if (P.kind == PK_FULL) DUSTB_COUNT(PK_FULL, 1);
        else DUSTB_COUNT(PK_IMEX, 1);
      } else {
        if (P.kind == PK_HALF) DUSTB_COUNT(PK_HALF, 0);
        else if (P.kind == PK_FULL) DUSTB_COUNT(PK_FULL, 0);
        else DUSTB_COUNT(PK_IMEX, 0);
      }
#undef DUSTB_COUNT
    }
    if ((rc = dustb_host::launch_status("mixed count"))) return rc;
  }
  {
    Scope sc(DUSTB_K_FILL, st);
    if ((rc = exclusive_scan(S.cstart, nbins(ncell), S.bsum, st))) return rc;
    cudaMemcpyAsync(S.cursor, S.cstart, 4 * (size_t)nbins(ncell), cudaMemcpyDeviceToDevice, st);
  }
  Scope sc(DUSTB_K_MOVE, st);
  if (n > 0) {
#define DUSTB_MOVE(K, SPF) k_move<K, SPF><<<nblk(n), kT, 0, st>>>(src, dst, S.key, S.cursor, G, n, P)
    if (G.ml) {
      if (P.kind == PK_HALF) DUSTB_MOVE(PK_HALF, 2);
      else if (P.kind == PK_FULL) DUSTB_MOVE(PK_FULL, 2);
      else DUSTB_MOVE(PK_IMEX, 2);
    } else if (G.ghost) {
      if (P.kind == PK_HALF) DUSTB_MOVE(PK_HALF, 1);
      else if (P.kind == PK_FULL) DUSTB_MOVE(PK_FULL, 1);
      else DUSTB_MOVE(PK_IMEX, 1);
    } else {
      if (P.kind == PK_HALF) DUSTB_MOVE(PK_HALF, 0);
      else if (P.kind == PK_FULL) DUSTB_MOVE(PK_FULL, 0);
      else DUSTB_MOVE(PK_IMEX, 0);
    }
#undef DUSTB_MOVE
  }
  return dustb_host::launch_status("mixed move");
}

}  // namespace

extern "C" {

long long dustb_mixed_workspace_bytes(const dustb_mesh *mesh, int npart) {
  if (!mesh) return -1;
  MState S;
  long long need = 0;
  carve(*mesh, npart, nullptr, 0, S, &need);
  return need;
}

int dustb_mixed_import(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws,
                       long long bytes, void *stream) {
  if (!params_ok(c, mp) || !rows_attached(c)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  Geo G = make_geo(c, mp);
  const int n = c->part.npart;
  const long long ncell = ncell_of(c->mesh);
  cudaMemsetAsync(S.head, 0, sizeof(MHead), st);   // the rows carry every kick so far
  cudaMemsetAsync(S.cstart, 0, 4 * (size_t)nbins(ncell), st);
  if (n > 0)
    k_import<<<nblk(n), kT, 0, st>>>(c->part.pr, c->part.pi, c->part.stride, n, S.B, S.cstart, G, c->err);
  int rc = exclusive_scan(S.cstart, nbins(ncell), S.bsum, st);
  if (rc) return rc;
  cudaMemcpyAsync(S.cursor, S.cstart, 4 * (size_t)nbins(ncell), cudaMemcpyDeviceToDevice, st);
  if (n > 0) k_sortmove<<<nblk(n), kT, 0, st>>>(S.B, S.A, n, S.cursor);
  return dustb_host::launch_status("mixed_import");
}

int dustb_mixed_export(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws,
                       long long bytes, void *stream) {
  if (!params_ok(c, mp) || !rows_attached(c)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  Geo G = make_geo(c, mp);
  const int n = c->part.npart;
  if (n > 0)
    k_export<<<nblk(n), kT, 0, (cudaStream_t)stream>>>(c->part.pr, c->part.pi, c->part.stride, n, S.A, G,
                                                        c->f.resid, S.head);
  return dustb_host::launch_status("mixed_export");
}

int dustb_mixed_sort(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws, long long bytes,
                     void *stream) {
  if (!params_ok(c, mp)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = c->part.npart;
  int rc = sort_into(S, S.A, S.B, c->mesh, n, st);
  if (rc) return rc;
  if (n > 0) k_copy_buf<<<nblk(n), kT, 0, st>>>(S.B, S.A, n);
  return dustb_host::launch_status("mixed_sort");
}

int dustb_mixed_tune(const dustb_ctx *c, dustb_mixed_params *mp, void *ws, long long bytes,
                     double a_dt, double *best_ms, void *stream) {
  if (!params_ok(c, mp) || !(a_dt > 0.0)) return DUSTB_EINVAL;
  if (!c->mesh.multi_d) return DUSTB_EUNSUP;
  const Geo G = make_geo(c, mp);
  if (!geo_ok(mp, G)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  if (g_timing.on) return DUSTB_EUNSUP;          // (its events would interleave)
  const int nx1 = c->mesh.nx1, nx2 = c->mesh.nx2;
  const int keep = mp->variant & ~DUSTB_MIXED_GRID_TILES;   // (the probe hook, the ledger flag)
  // the candidates: rows per tile (tiles of at most 256 cells), particles per pass (the
  // default, or passes sized for 2.25, 4 and 4.5 thousand particles), persistent CTAs on the
  // work queue or one CTA per tile
  struct Cand { int rows, chunk, grid; };
  std::vector<Cand> cands;
  for (int r : {1, 2, 4, 8})
    if (nx2 % r == 0 && r * nx1 <= kMaxTileThreads)
      for (int ch : {0, 2304, 4096, 4608})
        for (int g : {0, 1}) cands.push_back({r, ch, g});
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return DUSTB_ELAUNCH;
  float best = -1.0f;
  Cand pick{mp->rows_per_tile, mp->chunk, (mp->variant & DUSTB_MIXED_GRID_TILES) ? 1 : 0};
  int rc = DUSTB_OK;
  TileArgs base{};
  base.a_dt = a_dt; base.err = c->err; base.deposit = 1;
  rc = gather_window(S, G, c->mesh, c->f.ustar, base, st);
  for (size_t q = 0; q < cands.size() && rc == DUSTB_OK; ++q) {
    dustb_mixed_params t = *mp;
    t.rows_per_tile = cands[q].rows;
    t.chunk = cands[q].chunk;
    t.variant = keep | (cands[q].grid ? DUSTB_MIXED_GRID_TILES : 0);
    Cfg cf;
    if (!pick_cfg(c->mesh, &t, cf)) continue;     // (the shape does not fit shared memory)
    // the Q/P and operator tiles on the shadow as it stands: they write only the stage's
    // scratch fields (qdep, the centre mass, work), which every cycle rewrites before use
    auto trial = [&]() {
      TileArgs T = base;
      int r = build_queue(S, G, cf, T, st);
      if (r) return r;
      T.dfield = c->f.qdep; T.dnvar = 5; T.res = c->f.resid;
      if ((r = launch_tile<MODE_QP>(S, S.A, G, cf, T, st, Q_QP))) return r;
      T.gfield = c->f.ustar; T.dfield = c->f.work; T.dnvar = 3;
      return launch_tile<MODE_OP>(S, S.A, G, cf, T, st, Q_OP);
    };
    if ((rc = trial())) break;                     // warm-up (kernel attributes, caches)
    cudaEventRecord(e0, st);
    for (int rep = 0; rep < 2 && rc == DUSTB_OK; ++rep) rc = trial();
    cudaEventRecord(e1, st);
    if (rc) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) { rc = DUSTB_ELAUNCH; break; }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (best < 0.0f || ms < best) { best = ms; pick = cands[q]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (best < 0.0f) return DUSTB_EUNSUP;
  mp->rows_per_tile = pick.rows;
  mp->chunk = pick.chunk;
  mp->variant = keep | (pick.grid ? DUSTB_MIXED_GRID_TILES : 0);
  if (best_ms) *best_ms = 0.5 * best;
  return DUSTB_OK;
}

int dustb_mixed_timing(int enable) {
  g_timing.on = enable != 0;
  for (int k = 0; k < DUSTB_K_NKERNELS; ++k) g_timing.used[k] = 0;
  return DUSTB_OK;
}

int dustb_mixed_kernel_times(double *ms, int *launches, int n) {
  for (int k = 0; k < DUSTB_K_NKERNELS && k < n; ++k) {
    double tot = 0.0;
    const size_t u = g_timing.used[k];
    for (size_t e = 0; e + 1 < u; e += 2) {
      float t = 0.0f;
      cudaEventSynchronize(g_timing.ev[k][e + 1]);
      if (cudaEventElapsedTime(&t, g_timing.ev[k][e], g_timing.ev[k][e + 1]) == cudaSuccess) tot += t;
    }
    if (ms) ms[k] = tot;
    if (launches) launches[k] = (int)(u / 2);
    g_timing.used[k] = 0;
  }
  return DUSTB_OK;
}

int dustb_mixed_imex_cycle(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws,
                           long long bytes, const dustb_imex_coeffs *co, void *stream) {
  if (!params_ok(c, mp) || !co || !(co->dt > 0.0)) return DUSTB_EINVAL;
  if (!c->mesh.multi_d) return DUSTB_EUNSUP;                        // 1-D: FP64 form
  // (the implicit shear shift is the 3-D shearing box's: 2-D meshes take the FP64 form)
  if ((co->sh[0] != 0.0 || co->sh[1] != 0.0) && !c->mesh.three_d) return DUSTB_EUNSUP;
  const Geo G = make_geo(c, mp);
  if (!geo_ok(mp, G)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  Cfg cf;
  if (!pick_cfg(c->mesh, mp, cf)) return DUSTB_EUNSUP;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = c->part.npart;
  const long long ncell = ncell_of(c->mesh);
  Ind d = make_ind(c->mesh);
  const size_t fbytes = (size_t)d.cells() * d.nmb * sizeof(double);
  const double g = co->gamma, dt = co->dt;
  const double gam0[2] = {1.0, (2.0 * g - 1.0) / (2.0 * g * g)};
  const double gam1[2] = {0.0, 1.0 - (2.0 * g - 1.0) / (2.0 * g * g)};
  const double beta[2] = {g, 1.0 / (2.0 * g)};
  const double atw22 = (1.0 - 2.0 * g * g) / 2.0 / g;
  const double a_dt = g * dt;
  const int br = c->phys.back_reaction, cons = c->phys.consistent_gas;
  int rc;
#define RUN(x) do { rc = (x); if (rc) return rc; } while (0)
  for (int stage = 1; stage <= 2; ++stage) {
    // stage 1 moves the shadow from A to B, stage 2 back to A
    const PBuf &src = (stage == 1) ? S.A : S.B;
    const PBuf &cur = (stage == 1) ? S.B : S.A;
    {
      Scope sc(DUSTB_K_CELLS, st);
      if (stage == 1) cudaMemcpyAsync(c->f.u1, c->f.u0, fbytes * c->f.nvar_gas, cudaMemcpyDeviceToDevice, st);
      dustb_cells::gas_rk(c, gam0[stage - 1], gam1[stage - 1], st);
      if (stage == 2 && br) {
        // with the ledger, the rate's FP32 rounding the stage-1 kick tiles recorded follows the
        // gas rate in the same pass
        if (!(mp->variant & DUSTB_MIXED_NO_LEDGER))
          dustb_cells::history_field(c, c->f.work, atw22 * dt, st);
        else
          dustb_cells::history(c, atw22 * dt, st);
      }
    }
    PushArgs P{};
    P.kind = PK_IMEX;
    P.gam0 = (float)gam0[stage - 1]; P.gam1 = (float)gam1[stage - 1];
    P.atw_dt = (stage == 2) ? (float)(atw22 * dt) : 0.0f;
    P.bdt = (float)(beta[stage - 1] * dt);
    for (int a = 0; a < 3; ++a)
      P.bdx[a] = G.ml ? (float)(beta[stage - 1] * dt / G.dx[a])
                      : (float)(beta[stage - 1] * dt * G.inv_dx[a]);
    P.gy = 0.0f;
    P.shy = (float)(co->sh[stage - 1] * G.inv_dx[1]);
    P.a_dt = a_dt; P.stage2 = (stage == 2);
    P.sbox = c->phys.shearing_box; P.strat = c->phys.stratified;
    P.q = (float)c->phys.qshear; P.om = (float)c->phys.omega0;
    // stage 2: stage 1's consistent kick (this cycle's split); stage 1: the previous
    // cycle's stage-2 kick, if it left one pending
    P.res = (stage == 1 || (br && cons)) ? c->f.resid : nullptr;
    P.head = S.head;
    P.set_pending = (stage == 2 && br && cons);
    P.x3rem = mp->x3_removed;
    P.err = c->err;
    const bool ledger = br && !(mp->variant & DUSTB_MIXED_NO_LEDGER);
    if (ledger) {
      // the push's momentum ledger (FP64 coefficients of the gas's own RK combination)
      P.u0 = c->f.u0; P.u1 = c->f.u1; P.nvg = c->f.nvar_gas;
      P.g0 = gam0[stage - 1]; P.g1 = gam1[stage - 1];
      P.atw = (stage == 2) ? atw22 * dt : 0.0;
    }
    P.inv_adt = 1.0 / a_dt;
    RUN(push_sort(S, src, cur, G, n, ncell, P, st));
    if (stage == 1) cudaMemsetAsync(&S.head->pending, 0, sizeof(int), st);   // applied
    TileArgs T{};
    T.a_dt = a_dt; T.err = c->err; T.deposit = 1; T.shy = P.shy;
    RUN(build_queue(S, G, cf, T, st));                // the stage's tiles, heaviest first
    const bool shift = P.shy != 0.0f;
    if (br) {
      {
        Scope sc(DUSTB_K_DEPOSIT_QP, st);
        cudaMemsetAsync(c->f.qdep, 0, fbytes * 5, st);
        T.dfield = c->f.qdep; T.dnvar = 5; T.res = c->f.resid;
        RUN(launch_tile<MODE_QP>(S, cur, G, cf, T, st, Q_QP));
        if (shift) RUN(launch_shift_edge<MODE_QP>(S, cur, G, T, st));
      }
      Scope sc(DUSTB_K_CELLS, st);
      RUN(ghost_add_if(c, G, c->f.qdep, 5, st, mp));
    }
    // periodic meshes: the deposits go straight into the owners' active cells and the
    // gathers read ghost cells from their owners, so no ghost exchange is needed
    {
      Scope sc(DUSTB_K_CELLS, st);
      RUN(dustb_solve_ustar(c, st));
    }
    if (br && c->phys.drag_solver >= DUSTB_SOLVER_DC1) {
      const int nsw = (c->phys.drag_solver == DUSTB_SOLVER_DC2) ? 2 : 1;
      for (int w = 0; w < nsw; ++w) {
        { Scope sc(DUSTB_K_CELLS, st);
          RUN(ghost_copy_if(c, G, c->f.ustar, st, mp)); }
        cudaMemsetAsync(c->f.work, 0, fbytes * 3, st);
        RUN(gather_window(S, G, c->mesh, c->f.ustar, T, st));
        { Scope sc(DUSTB_K_OPERATOR, st);
          T.gfield = c->f.ustar; T.dfield = c->f.work; T.dnvar = 3;
          RUN(launch_tile<MODE_OP>(S, cur, G, cf, T, st, Q_OP + w));
          if (shift) RUN(launch_shift_edge<MODE_OP>(S, cur, G, T, st)); }
        { Scope sc(DUSTB_K_CELLS, st);
          RUN(ghost_add_if(c, G, c->f.work, 3, st, mp));
          dustb_cells::dc_correct(c, st); }
      }
    }
    {
      Scope sc(DUSTB_K_CELLS, st);
      RUN(ghost_copy_if(c, G, c->f.ustar, st, mp));
    }
    if (br) cudaMemsetAsync(c->f.dmom, 0, fbytes * 3, st);
    // stage 1: the kick tiles record the rate's rounding in work for stage 2's history term
    // (work is free from here: the operator sweeps are done)
    if (ledger && stage == 1) cudaMemsetAsync(c->f.work, 0, fbytes * 3, st);
    RUN(gather_window(S, G, c->mesh, c->f.ustar, T, st));
    {
      Scope sc(DUSTB_K_KICK, st);
      T.gfield = c->f.ustar; T.dfield = c->f.dmom; T.dnvar = 3; T.deposit = br;
      T.ledger = ledger;
      T.hfield = (ledger && stage == 1) ? c->f.work : nullptr;
      RUN(launch_tile<MODE_KICK>(S, cur, G, cf, T, st, Q_KICK));
      if (shift) RUN(launch_shift_edge<MODE_KICK>(S, cur, G, T, st));
    }
    if (br) {
      Scope sc(DUSTB_K_CELLS, st);
      RUN(ghost_add_if(c, G, c->f.dmom, 3, st, mp));
      if (cons) dustb_cells::consistent_gas(c, a_dt, st);
      else dustb_cells::pmbr(c, a_dt, st);
      // stage 2's consistent dust kick is left pending (recorded by stage 2's count): the
      // next cycle's stage-1 push, or an export, applies it
    }
  }
  {
    // the gas tail's ghost exchange of the conserved state, once per cycle (nothing in the
    // drag step reads u0's ghost cells between the stages)
    Scope sc(DUSTB_K_CELLS, st);
    if (G.ml) RUN(dustb_ghost_copy_ml(c, c->f.u0, c->f.nvar_gas, mp->coarse, mp->coarse_bytes, st));
    else RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, st));
  }
  return DUSTB_OK;
}

int dustb_mixed_pc2_cycle(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws,
                          long long bytes, double dt, double *chi_max, void *stream) {
  if (!params_ok(c, mp) || !(dt > 0.0)) return DUSTB_EINVAL;
  if (!c->mesh.multi_d) return DUSTB_EUNSUP;                        // 1-D: FP64 form
  if (c->mesh.nghbr_ml) return DUSTB_EUNSUP;                        // (refined: imex only)
  const Geo G = make_geo(c, mp);
  if (!geo_ok(mp, G)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  Cfg cf;
  if (!pick_cfg(c->mesh, mp, cf)) return DUSTB_EUNSUP;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = c->part.npart;
  const long long ncell = ncell_of(c->mesh);
  Ind d = make_ind(c->mesh);
  const size_t fbytes = (size_t)d.cells() * d.nmb * sizeof(double);
  const double h = 0.5 * dt;
  const int br = c->phys.back_reaction;
  int rc;
  // FirstTwoImpRK's gas register and the gas stand-in's first stage
  {
    Scope sc(DUSTB_K_CELLS, st);
    cudaMemcpyAsync(c->f.u1, c->f.u0, fbytes * c->f.nvar_gas, cudaMemcpyDeviceToDevice, st);
    dustb_cells::gas_rk(c, 1.0, 0.0, st);
  }
  TileArgs T{};
  T.a_dt = h; T.err = c->err; T.deposit = 1;
  T.pc = make_pc2(c, G, dt);
  if (br) {
    // the predictor: the old gas velocity m/rho of u1 (work), the tiles' deposits into
    // qdep 1..4, the exchange, the stiffness damping and the gas update
    {
      Scope sc(DUSTB_K_CELLS, st);
      const long long per = d.cells(), tot = per * d.nmb;
      k_gas_velocity<<<nblk(tot), kT, 0, st>>>(c->f.u1, c->f.nvar_gas, c->f.work, per, tot);
      RUN(dustb_host::launch_status("mixed gas velocity"));
    }
    RUN(gather_window(S, G, c->mesh, c->f.work, T, st));
    {
      Scope sc(DUSTB_K_DEPOSIT_QP, st);
      cudaMemsetAsync(c->f.qdep, 0, fbytes * 5, st);
      T.gfield = c->f.work; T.dfield = c->f.qdep + d.cells(); T.dnvar = 5;
      RUN(build_queue(S, G, cf, T, st));             // the tiles of copy A
      RUN(launch_tile<MODE_PRED>(S, S.A, G, cf, T, st, Q_PRED));
    }
    Scope sc(DUSTB_K_CELLS, st);
    RUN(ghost_add_if(c, G, c->f.qdep, 5, st, mp));
    RUN(dustb_pc2_apply_predictor(c, dt, chi_max, st));
  }
  {
    // the gas tail: exchange, the midpoint u* (every cell), the stand-in's second stage
    Scope sc(DUSTB_K_CELLS, st);
    RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, st));
    RUN(dustb_pc2_midpoint(c, st));
    dustb_cells::gas_rk(c, 0.5, 0.5, st);
  }
  // the half step: A -> B sorted by the cell of each particle's gather position
  PushArgs P{};
  P.kind = PK_HALF;
  P.gam0 = 1.0f; P.gam1 = 0.0f; P.atw_dt = 0.0f; P.bdt = 0.0f;
  for (int a = 0; a < 3; ++a) P.bdx[a] = T.pc.hdx[a];
  P.gy = T.pc.gy;
  P.sdy = (float)(c->phys.qshear * c->phys.omega0 * dt * G.inv_dx[1]);
  P.a_dt = h; P.stage2 = 0;
  P.sbox = c->phys.shearing_box; P.strat = c->phys.stratified;
  P.q = (float)c->phys.qshear; P.om = (float)c->phys.omega0;
  P.res = nullptr; P.head = S.head; P.set_pending = 0;
  P.x3rem = mp->x3_removed; P.err = c->err;
  RUN(push_sort(S, S.A, S.B, G, n, ncell, P, st));
  if (br) cudaMemsetAsync(c->f.dmom, 0, fbytes * 3, st);
  RUN(gather_window(S, G, c->mesh, c->f.ustar, T, st));
  {
    Scope sc(DUSTB_K_KICK, st);
    T.gfield = c->f.ustar; T.dfield = c->f.dmom; T.dnvar = 3; T.deposit = br;
    RUN(build_queue(S, G, cf, T, st));               // the tiles of copy B (half step)
    RUN(launch_tile<MODE_ADV>(S, S.B, G, cf, T, st, Q_ADV));
    if (G.ghost && n > 0) {
      T.cstart = S.cstart;
      if (G.scheme == 2) k_pc2_edge<2><<<148 * 4, kT, 0, st>>>(S.B, G, T);
      else if (G.scheme == 1) k_pc2_edge<1><<<148 * 4, kT, 0, st>>>(S.B, G, T);
      else k_pc2_edge<0><<<148 * 4, kT, 0, st>>>(S.B, G, T);
      RUN(dustb_host::launch_status("mixed pc2 edge"));
    }
  }
  // the move to the new position: B -> A sorted by cell (routing as SetNewPrtclGID)
  P.kind = PK_FULL;
  P.gam0 = 0.0f; P.gam1 = 1.0f;
  for (int a = 0; a < 3; ++a) P.bdx[a] = 0.0f;
  P.gy = 0.0f;
  RUN(push_sort(S, S.B, S.A, G, n, ncell, P, st));
  if (br) {
    Scope sc(DUSTB_K_CELLS, st);
    RUN(ghost_add_if(c, G, c->f.dmom, 3, st, mp));
    RUN(dustb_pc2_commit(c, 0.5, st));
  }
  {
    Scope sc(DUSTB_K_CELLS, st);
    RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, st));
  }
#undef RUN
  return DUSTB_OK;
}

}  // extern "C"
