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
#include <vector>

#include "dustb_common.cuh"
#include "dustb_sort.cuh"

namespace dustb_cells {
void gas_rk(const dustb_ctx *c, double g0, double g1, cudaStream_t st);
void history(const dustb_ctx *c, double atw_dt, cudaStream_t st);
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

struct MState {
  MHead *head;
  PBuf A, B;                     // A holds the shadow between cycles
  int *key;                      // new cell of each particle (count -> move)
  int *cstart, *cursor, *bsum;
};

struct Geo {
  int nmb, nx1, nx2, nx3, three_d, gids;
  int l1, l2, l3;              // log2 of nx1, nx2, nx3 when all are powers of two, else -1
  int n1, n2, n3, is, js, ks;
  long long vstride;           // cells of one variable of one block
  const int *nghbr;
  const double *mb;
  double dx[3], inv_dx[3], vol;
  int scheme;
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
  const size_t o_key = off; off += al256(4 * N);
  const size_t o_cs = off; off += al256(4 * (size_t)(ncell + 1));
  const size_t o_cur = off; off += al256(4 * (size_t)(ncell + 1));
  const size_t o_bs = off; off += al256(4 * (size_t)scan_bsum_ints(ncell + 1));
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
// orders this thread's earlier ordinary shared-memory accesses before later bulk copies
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// bounded wait for the barrier's phase; false (and the error bit) if it never completes
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned *err) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try_wait(bar, parity)) return true;
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
    if (ig < 0 || ig >= nx[a]) { report(err, DUSTB_ERR_HALO); ig = ig < 0 ? 0 : nx[a] - 1; }
    float fo = (float)(cell - (double)ig);
    if (!(fo >= 0.0f)) fo = 0.0f;
    if (fo >= 1.0f) fo = 0.99999994f;
    ic[a] = ig; of[a] = fo;
    dd[a] = (float)((x1[a] - x[a]) * G.inv_dx[a]);
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
// cycle is applied to the exported velocities and rates (rounded as the next push would)
__global__ void k_export(double *pr, int *pi, long long stride, int n, PBuf A, Geo G,
                         const double *res, const MHead *head) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int m, k, j, i;
  decode(G, A.cell[q], m, k, j, i);
  const int p = A.pid[q];
  float vel[3] = {A.f[F_VX][q], A.f[F_VY][q], A.f[F_VZ][q]};
  float rate[3] = {A.f[F_RX][q], A.f[F_RY][q], A.f[F_RZ][q]};
  if (res && head->pending && A.f[F_M][q] > 0.0f) {
    const long long b = G.at(m, 4, 0, k + G.ks, j + G.js, i + G.is);
    const double cj = (double)A.f[F_CC][q];
    for (int a = 0; a < 3; ++a) {
      const double d = __dmul_rn(cj, res[b + a * G.vstride]);
      vel[a] = __fadd_rn(vel[a], __double2float_rn(d));
      rate[a] += (float)(d / head->a_dt);
    }
  }
  auto W = [&](int r, double v) { pr[(long long)r * stride + p] = v; };
  const double *sz = G.mb + (long long)m * 9;
  const double x = sz[X1MIN] + ((double)i + (double)A.f[F_OX][q]) * G.dx[0];
  const double y = sz[X2MIN] + ((double)j + (double)A.f[F_OY][q]) * G.dx[1];
  W(DUSTB_IPX, x); W(DUSTB_IPY, y);
  W(DUSTB_IPX1, x + (double)A.f[F_AX][q] * G.dx[0]);
  W(DUSTB_IPY1, y + (double)A.f[F_AY][q] * G.dx[1]);
  if (G.three_d) {
    const double z = sz[X3MIN] + ((double)k + (double)A.f[F_OZ][q]) * G.dx[2];
    W(DUSTB_IPZ, z);
    W(DUSTB_IPZ1, z + (double)A.f[F_AZ][q] * G.dx[2]);
  }
  W(DUSTB_IPVX, vel[0]); W(DUSTB_IPVY, vel[1]); W(DUSTB_IPVZ, vel[2]);
  W(DUSTB_IPVX1, A.f[F_WX][q]); W(DUSTB_IPVY1, A.f[F_WY][q]); W(DUSTB_IPVZ1, A.f[F_WZ][q]);
  W(DUSTB_IPRX, rate[0]); W(DUSTB_IPRY, rate[1]); W(DUSTB_IPRZ, rate[2]);
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
struct PushArgs {
  float gam0, gam1, atw_dt;
  float bdt;                  // beta*dt (velocity kick)
  float bdx[3];               // beta*dt/dx per axis (drift in cells)
  double a_dt;
  int stage2;
  int sbox, strat;
  float q, om;
  // the consistent split's dust kick folded into the push: stage 2 applies stage 1's kick
  // (res = stage 1's dust residual); stage 1 applies the previous cycle's stage-2 kick when
  // head->pending is set (res = that residual)
  const double *res;
  MHead *head;
  int set_pending;            // stage 2: record this cycle's stage-2 kick as pending
  unsigned *err;
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

// the new position: the drift of ExplicitPush (src/dust/dust_push.cpp:289-296) in cell units,
// x <- x + gam1 (x1 - x) + beta dt xdot (gam0 + gam1 = 1), and the cell carry that replaces
// SetNewPrtclGID (the neighbour in the crossing direction; periodic images are neighbours).
// Every operation is explicitly rounded: count and move must agree bit for bit.
__device__ __forceinline__ int advance(const Geo &G, const PushArgs &P, int &m, int &k, int &j,
                                       int &i, float o[3], float d1[3], const float v[3]) {
  float xsh = 0.0f;
  if (P.sbox && G.three_d) {
    const double *sz = G.mb + (long long)m * 9;
    const double x = __dadd_rn(sz[X1MIN], __dmul_rn(__dadd_rn((double)i, (double)o[0]), G.dx[0]));
    xsh = __fmul_rn(__fmul_rn(P.q, P.om), __double2float_rn(x));
  }
  const float xdot[3] = {v[0], __fsub_rn(v[1], xsh), v[2]};
  const int nax = G.three_d ? 3 : 2;
  int c[3] = {0, 0, 0};
  for (int a = 0; a < nax; ++a) {
    const float s = __fmaf_rn(P.bdx[a], xdot[a], __fmul_rn(P.gam1, d1[a]));
    o[a] = __fadd_rn(o[a], s);
    d1[a] = __fsub_rn(d1[a], s);
    int ci = (int)floorf(o[a]);
    o[a] = __fsub_rn(o[a], (float)ci);
    if (o[a] >= 1.0f) { o[a] = __fsub_rn(o[a], 1.0f); ++ci; }
    c[a] = ci;
  }
  i += c[0]; j += c[1]; k += c[2];
  const int o1 = (i < 0) ? -1 : ((i >= G.nx1) ? 1 : 0);
  const int o2 = (j < 0) ? -1 : ((j >= G.nx2) ? 1 : 0);
  const int o3 = (k < 0) ? -1 : ((k >= G.nx3) ? 1 : 0);
  if (o1 | o2 | o3) {
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
  }
  return encode(G, m, k, j, i);
}

// count: the new cell of every particle and the per-cell histogram
__global__ void __launch_bounds__(kT) k_count(PBuf S, int *key_out, int *count, Geo G, int n,
                                              PushArgs P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  int m, k, j, i;
  decode(G, S.cell[p], m, k, j, i);
  float o[3] = {S.f[F_OX][p], S.f[F_OY][p], S.f[F_OZ][p]};
  float v[3] = {S.f[F_VX][p], S.f[F_VY][p], S.f[F_VZ][p]};
  float d1[3] = {0.0f, 0.0f, 0.0f};
  if (P.stage2) { d1[0] = S.f[F_AX][p]; d1[1] = S.f[F_AY][p]; d1[2] = S.f[F_AZ][p]; }
  if (P.res && (P.stage2 || P.head->pending) && S.f[F_M][p] > 0.0f) {
    double d[3];
    consistent_dv(G, P, S.f[F_CC][p], m, k, j, i, d);
    for (int a = 0; a < 3; ++a) v[a] = __fadd_rn(v[a], __double2float_rn(d[a]));
  }
  const int key = advance(G, P, m, k, j, i, o, d1, v);
  key_out[p] = key;
  warp_count(count, key, act);
  if (P.set_pending && p == 0) { P.head->a_dt = P.a_dt; P.head->pending = 1; }
}

// move: the whole push of every particle, written to its slot in dst
__global__ void __launch_bounds__(kT) k_move(PBuf S, PBuf D, const int *key_in, int *cursor,
                                             Geo G, int n, PushArgs P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < n;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  const int key = key_in[p];
  const int q = warp_slot(cursor, key, act);
  int m, k, j, i;
  decode(G, S.cell[p], m, k, j, i);
  float o[3] = {S.f[F_OX][p], S.f[F_OY][p], S.f[F_OZ][p]};
  float v[3] = {S.f[F_VX][p], S.f[F_VY][p], S.f[F_VZ][p]};
  const float ts = S.f[F_TS][p], mass = S.f[F_M][p];
  // (the rates: stage 1's velocity does not use them and every stage's kick rewrites them)
  const bool kick = P.res && (P.stage2 || P.head->pending);
  float cc = (P.stage2 || kick) ? S.f[F_CC][p] : 0.0f;
  float v1[3], d1[3], r[3] = {0.0f, 0.0f, 0.0f};
  if (P.stage2) { r[0] = S.f[F_RX][p]; r[1] = S.f[F_RY][p]; r[2] = S.f[F_RZ][p]; }
  if (kick && mass > 0.0f) {
    double d[3];
    consistent_dv(G, P, cc, m, k, j, i, d);
    for (int a = 0; a < 3; ++a) {
      v[a] = __fadd_rn(v[a], __double2float_rn(d[a]));
      r[a] += (float)(d[a] / P.a_dt);
    }
  }
  if (P.stage2) {
    v1[0] = S.f[F_WX][p]; v1[1] = S.f[F_WY][p]; v1[2] = S.f[F_WZ][p];
    d1[0] = S.f[F_AX][p]; d1[1] = S.f[F_AY][p]; d1[2] = S.f[F_AZ][p];
  } else {
    // FirstTwoImpRK: (x1, v1) <- (x, v); the drag factor of the cycle, formed in FP64
    v1[0] = v[0]; v1[1] = v[1]; v1[2] = v[2];
    d1[0] = d1[1] = d1[2] = 0.0f;
    cc = (float)(P.a_dt / ((double)ts + P.a_dt));
  }
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
  const float atw = P.stage2 ? P.atw_dt : 0.0f;
  const float nv[3] = {P.gam0 * v[0] + P.gam1 * v1[0] + P.bdt * fx + atw * r[0],
                       P.gam0 * v[1] + P.gam1 * v1[1] + P.bdt * fy + atw * r[1],
                       P.gam0 * v[2] + P.gam1 * v1[2] + P.bdt * fz + atw * r[2]};
  const int key2 = advance(G, P, m, k, j, i, o, d1, v);
  if (key2 != key) report(P.err, DUSTB_ERR_WINDOW);   // count and move disagree: never expected
  D.cell[q] = key; D.pid[q] = S.pid[p];
  D.f[F_OX][q] = o[0]; D.f[F_OY][q] = o[1]; D.f[F_OZ][q] = o[2];
  D.f[F_VX][q] = nv[0]; D.f[F_VY][q] = nv[1]; D.f[F_VZ][q] = nv[2];
  D.f[F_AX][q] = d1[0]; D.f[F_AY][q] = d1[1]; D.f[F_AZ][q] = d1[2];
  D.f[F_WX][q] = v1[0]; D.f[F_WY][q] = v1[1]; D.f[F_WZ][q] = v1[2];
  // (no rates: the kick tile of this stage writes every particle's rate)
  D.f[F_TS][q] = ts; D.f[F_M][q] = mass; D.f[F_CC][q] = cc;
}

// ---- tile deposit kernels -------------------------------------------------------------------
enum { MODE_QP = 0, MODE_OP = 1, MODE_KICK = 2 };

struct TileArgs {
  int tj, chunk, tpp;          // rows per tile, buffer columns, tiles per (block, plane)
  double a_dt;
  const int *cstart;           // cell -> particle ranges of the sorted shadow
  const double *gfield;        // gather field (3 vars), MODE_OP / MODE_KICK
  double *dfield;              // deposit field
  int dnvar;
  double *res;                 // MODE_QP: resid, the centre mass goes to var 3
  int deposit;                 // 0: kick only (no back-reaction)
  unsigned *err;
};

// shared rows of a tile pass: the copied fields, then (operator, kick) the per-particle
// values of the gather phase in rows 5..7
constexpr int kTileRows = 8;

// the index of variable 0 of block-local cell (kk, jj, ii) of block m in a field of nvar
// variables, or -1 if no block owns it; a cell one beyond the block maps to the owning
// neighbour's active cell (the ghost exchanges folded into the index)
__device__ __forceinline__ long long cell_at(const Geo &G, int m, int nvar, int kk, int jj, int ii) {
  int mo;
  if (!G.owner(m, kk, jj, ii, mo)) return -1;
  return G.at(mo, nvar, 0, G.ks + kk, G.js + jj, G.is + ii);
}
__device__ __forceinline__ float2 dup(float x) { return make_float2(x, x); }

// the 27-point sums of one source cell's particles: values 0, 1 as a packed pair; values 2, 3
// as a pair (Q/P) or value 2 alone (operator, kick)
template <int MODE, int D3>
struct CellSums {
  static constexpr int WK = D3 ? 3 : 1;
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
          if (MODE == MODE_QP) a23[c][b][a] = make_float2(0.0f, 0.0f);
          else a2[c][b][a] = 0.0f;
        }
  }
  __device__ __forceinline__ float val(int c, int b, int a, int q) const {
    return q == 0 ? a01[c][b][a].x : q == 1 ? a01[c][b][a].y
         : (MODE == MODE_QP ? (q == 2 ? a23[c][b][a].x : a23[c][b][a].y) : a2[c][b][a]);
  }
  // sum_cba += wz_c wy_b (wx_a q): the x weights folded into the values first
  __device__ __forceinline__ void add(const float wx[3], const float wy[3], const float wz[3],
                                      float2 q01, float2 q23) {
    float2 s01[3], s23[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      s01[a] = __fmul2_rn(dup(wx[a]), q01);
      if (MODE == MODE_QP) s23[a] = __fmul2_rn(dup(wx[a]), q23);
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
          if (MODE == MODE_QP) a23[c][b][a] = __ffma2_rn(dup(wzy), s23[a], a23[c][b][a]);
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
  __device__ __forceinline__ void load(const Geo &G, const double *f, int m, int k, int jrow,
                                       int ci) {
#pragma unroll
    for (int c = 0; c < WK; ++c)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        // this cell's column of the (c, b) row; its x neighbours are the next words unless
        // the cell ends the block's row
        const int kk = D3 ? k - 1 + c : 0, jj = jrow - 1 + b;
        const long long rb = cell_at(G, m, 3, kk, jj, ci);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          long long at = (rb >= 0) ? rb + (a - 1) : -1;
          if ((a == 0 && ci == 0) || (a == 2 && ci == G.nx1 - 1)) at = cell_at(G, m, 3, kk, jj, ci - 1 + a);
          xy[c][b][a] = make_float2(0.0f, 0.0f);
          z[c][b][a] = 0.0f;
          if (at >= 0) {
            xy[c][b][a] = make_float2((float)f[at], (float)f[at + G.vstride]);
            z[c][b][a] = (float)f[at + 2 * G.vstride];
          }
        }
      }
  }
  // u = sum over (c, b) of wz_c wy_b (sum over a of wx_a g_cba)
  __device__ __forceinline__ void gather(const float wx[3], const float wy[3], const float wz[3],
                                         float2 &uxy, float &uz) const {
    uxy = make_float2(0.0f, 0.0f);
    uz = 0.0f;
#pragma unroll
    for (int c = 0; c < WK; ++c) {
      const float wzc = D3 ? wz[c] : 1.0f;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        float2 txy = __fmul2_rn(dup(wx[0]), xy[c][b][0]);
        float tz = wx[0] * z[c][b][0];
#pragma unroll
        for (int a = 1; a < 3; ++a) {
          txy = __ffma2_rn(dup(wx[a]), xy[c][b][a], txy);
          tz = fmaf(wx[a], z[c][b][a], tz);
        }
        const float wzy = wzc * wy[b];
        uxy = __ffma2_rn(dup(wzy), txy, uxy);
        uz = fmaf(wzy, tz, uz);
      }
    }
  }
};

// the sums of every source cell of the tile, staged in shared memory as float4 (values 0..3)
// at [(c*3 + b)*3 + a][cell], for the window pass below
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
                        MODE == MODE_QP ? A.val(c, b, a, 3) : 0.0f);
}

// adds the tile's deposit window to the FP64 field, one add per window cell and value: a
// window cell (z plane c, row wy, column wx) sums the staged contributions of the up to 9
// source cells of its plane that reach it; window cells beyond the block go to the owning
// neighbour's active cell (the additive ghost exchange folded into the add)
template <int MODE, int D3>
__device__ __forceinline__ void add_window(const float4 *s_acc, const Geo &G, const TileArgs &T,
                                           int m, int k, int j0, int tj) {
  constexpr int NC = (MODE == MODE_QP) ? 4 : 3;
  constexpr int WK = D3 ? 3 : 1;
  const int nx1 = G.nx1, nct = tj * nx1;
  const int WI = nx1 + 2, WJ = tj + 2, nplane = WJ * WI;
  for (int t = threadIdx.x; t < WK * nplane; t += blockDim.x) {
    const int c = t / nplane, rem = t - c * nplane;
    const int wy = rem / WI, wx = rem - wy * WI;
    const long long at = cell_at(G, m, T.dnvar, D3 ? k - 1 + c : 0, j0 - 1 + wy, wx - 1);
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
        const float4 v = s_acc[((c * 3 + b) * 3 + a) * nct + cj * nx1 + ci];
        s.x += v.x; s.y += v.y; s.z += v.z; s.w += v.w;
      }
    }
    double *f = T.dfield + at;
    if (s.x != 0.0f) atomicAdd(f, (double)s.x);
    if (s.y != 0.0f) atomicAdd(f + G.vstride, (double)s.y);
    if (s.z != 0.0f) atomicAdd(f + 2 * G.vstride, (double)s.z);
    if (NC > 3 && s.w != 0.0f) atomicAdd(f + 3 * G.vstride, (double)s.w);
  }
}

// One CTA per tile of tj rows of one plane, one thread per source cell.  Q/P: the sums of a
// cell's particles are kept in registers over all passes.  Operator and kick: per pass, a
// gather phase (the 27 gather values in registers) writes each particle's deposit value (or
// velocity change) into its column, then a deposit phase sums them and adds them to the
// field; the gather values and the sums are never live together.
template <int MODE, int D3, int SCHEME>
__global__ void __launch_bounds__(kMaxTileThreads, 1) k_tile(PBuf S, Geo G, TileArgs T) {
  constexpr int NF = (MODE == MODE_OP) ? 5 : 8;    // fields copied: ox oy oz cc m [vx vy vz]
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  const int nx1 = G.nx1, tj = T.tj;
  const int nct = tj * nx1;                        // source cells of the tile = threads
  int t = blockIdx.x;
  const int per_block = G.nx3 * T.tpp;
  const int m = t / per_block;
  t -= m * per_block;
  const int k = t / T.tpp;
  const int j0 = (t - k * T.tpp) * tj;
  const int c0 = encode(G, m, k, j0, 0);
  const int CH = T.chunk;                          // buffer columns (multiple of 4)
  int *s_cs = (int *)smem;                         // [nct + 1] cell ranges
  float *s_f = (float *)(smem + (((size_t)(nct + 1) * 4 + 15) & ~(size_t)15));  // [8][CH]
  float4 *s_acc = (float4 *)s_f;                   // the staged sums, after the rows
  const int cl = threadIdx.x;                      // this thread's source cell
  const int cj_l = cl / nx1, ci_l = cl - cj_l * nx1;
  const int jrow = j0 + cj_l;

  const int CHP = CH - 8;                          // particles per pass (room to round out)
  // the particle range [cb, ce) of a pass, field by field, rounded out to 16-byte groups
  auto issue_pass = [&](int cb, int ce) {
    const int a0 = cb & ~3, a1 = (ce + 3) & ~3;
    const unsigned bytes = (unsigned)(a1 - a0) * 4u;
    const int fl[8] = {F_OX, F_OY, F_OZ, F_CC, F_M, F_VX, F_VY, F_VZ};
    fence_proxy_async();
    mbar_arrive_tx(&bar, bytes * NF);
#pragma unroll
    for (int f = 0; f < NF; ++f) bulk_copy(s_f + f * CH, S.f[fl[f]] + a0, bytes, &bar);
  };
  if (threadIdx.x == 0) {
    // the first pass's copies go out before the cell ranges are read
    mbar_init(&bar, 1);
    const int p0 = T.cstart[c0], p1 = T.cstart[c0 + nct];
    if (p1 > p0) issue_pass(p0, min(p1, p0 + CHP));
  }
  for (int x = threadIdx.x; x <= nct; x += blockDim.x) s_cs[x] = T.cstart[c0 + x];
  __syncthreads();
  const int P0 = s_cs[0], P1 = s_cs[nct];
  const int c_lo = s_cs[cl], c_hi = s_cs[cl + 1];  // this cell's particles
  CellSums<MODE, D3> qp;                           // Q/P: kept over all passes
  if (MODE == MODE_QP) qp.zero();
  float qt = 0.0f;
  const float inv_vol = (float)(1.0 / G.vol);
  const float inv_adt = (float)(1.0 / T.a_dt);
  unsigned parity = 0;

  for (int cb = P0; cb < P1; cb += CHP) {
    const int ce = min(P1, cb + CHP), cnt = ce - cb;
    const int a0 = cb & ~3, sh = cb - a0;
    if (threadIdx.x == 0 && cb != P0) issue_pass(cb, ce);
    GatherWindow<D3> win;
    if (MODE != MODE_QP) win.load(G, T.gfield, m, k, jrow, ci_l);   // while the copies fly
    const bool ok = mbar_wait(&bar, parity, T.err);
    parity ^= 1u;
    if (__syncthreads_or(!ok)) {
      // the copies never completed: wait once more (bounded) for them, then give up the tile
      mbar_wait(&bar, parity ^ 1u, T.err);
      return;
    }
    // this cell's particles in the pass, at columns lo..hi of the rows
    const int lo = max(c_lo, cb) - a0, hi = min(c_hi, ce) - a0;
    if (MODE == MODE_QP) {
      for (int r = lo; r < hi; ++r) {
        float wx_[3], wy_[3], wz_[3];
        wts(SCHEME, s_f[r], wx_);
        wts(SCHEME, s_f[CH + r], wy_);
        if (D3) wts(SCHEME, s_f[2 * CH + r], wz_);
        const float mc = s_f[4 * CH + r] * s_f[3 * CH + r] * inv_vol;
        qt += mc;
        qp.add(wx_, wy_, wz_, make_float2(mc, mc * s_f[5 * CH + r]),
               make_float2(mc * s_f[6 * CH + r], mc * s_f[7 * CH + r]));
      }
    } else {
      // gather phase: the operator's m c u / V, or the kick's velocity change, into rows 5..7
      for (int r = lo; r < hi; ++r) {
        float wx_[3], wy_[3], wz_[3];
        wts(SCHEME, s_f[r], wx_);
        wts(SCHEME, s_f[CH + r], wy_);
        if (D3) wts(SCHEME, s_f[2 * CH + r], wz_);
        float2 uxy;
        float uz;
        win.gather(wx_, wy_, wz_, uxy, uz);
        const float c32 = s_f[3 * CH + r];
        if (MODE == MODE_OP) {
          const float mc = s_f[4 * CH + r] * c32 * inv_vol;
          s_f[5 * CH + r] = mc * uxy.x; s_f[6 * CH + r] = mc * uxy.y; s_f[7 * CH + r] = mc * uz;
        } else {
          // GatherKickPMBR (src/dust/dust_pm.cpp:534-563): the applied velocity change
          const float vx = s_f[5 * CH + r], vy = s_f[6 * CH + r], vz = s_f[7 * CH + r];
          s_f[5 * CH + r] = (vx + c32 * (uxy.x - vx)) - vx;
          s_f[6 * CH + r] = (vy + c32 * (uxy.y - vy)) - vy;
          s_f[7 * CH + r] = (vz + c32 * (uz - vz)) - vz;
        }
      }
      if (MODE == MODE_KICK) {
        // the kicked velocities and rates of the pass, particle by particle (coalesced):
        // v <- v + dv, R <- dv / a_dt
        __syncthreads();
        // (four particles per thread at a time, their velocity loads issued together)
        constexpr int U = 4;
        for (int x0 = threadIdx.x; x0 < cnt; x0 += U * blockDim.x) {
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
            const float dvx = s_f[5 * CH + s], dvy = s_f[6 * CH + s], dvz = s_f[7 * CH + s];
            S.f[F_VX][p] = v[u][0] + dvx; S.f[F_VY][p] = v[u][1] + dvy; S.f[F_VZ][p] = v[u][2] + dvz;
            S.f[F_RX][p] = dvx * inv_adt; S.f[F_RY][p] = dvy * inv_adt; S.f[F_RZ][p] = dvz * inv_adt;
          }
        }
      }
      if (T.deposit) {
        // deposit phase: the sums of the values of this pass, added to the field
        CellSums<MODE, D3> sums;
        sums.zero();
        for (int r = lo; r < hi; ++r) {
          float wx_[3], wy_[3], wz_[3];
          wts(SCHEME, s_f[r], wx_);
          wts(SCHEME, s_f[CH + r], wy_);
          if (D3) wts(SCHEME, s_f[2 * CH + r], wz_);
          const float f = (MODE == MODE_OP) ? 1.0f : -s_f[4 * CH + r] * inv_vol;
          sums.add(wx_, wy_, wz_, make_float2(f * s_f[5 * CH + r], f * s_f[6 * CH + r]),
                   make_float2(f * s_f[7 * CH + r], 0.0f));
        }
        // the rows are read by now: their space takes the staged sums
        __syncthreads();
        stage_sums<MODE, D3>(sums, s_acc, cl, nct);
        __syncthreads();
        add_window<MODE, D3>(s_acc, G, T, m, k, j0, tj);
      }
    }
    // the next pass's copies overwrite the rows
    __syncthreads();
  }
  if (MODE == MODE_QP) {
    // centre mass m c / V of the cell (dust_imex_point_center_mass): only this cell's
    // particles have it as their centre, so it is stored, not added
    T.res[G.at(m, 4, 3, G.ks + k, G.js + jrow, G.is + ci_l)] = (double)qt;
    stage_sums<MODE, D3>(qp, s_acc, cl, nct);
    __syncthreads();
    add_window<MODE, D3>(s_acc, G, T, m, k, j0, tj);
  }
}

// shared memory of a tile: the cell ranges, then the larger of the pass rows and the staged
// sums (27 float4 per cell in 3-D, 9 in 2-D)
size_t tile_smem(int three_d, int tj, int nx1, int chunk) {
  const int nct = tj * nx1;
  const size_t rows = (size_t)kTileRows * chunk * 4;
  const size_t sums = (size_t)(three_d ? 27 : 9) * nct * 16;
  return (((size_t)(nct + 1) * 4 + 15) & ~(size_t)15) + (rows > sums ? rows : sums);
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
};

bool pick_cfg(const dustb_mesh &ms, const dustb_mixed_params *mp, Cfg &cf) {
  const int nx1 = ms.nx1, nx2 = ms.multi_d ? ms.nx2 : 1;
  if (mp->variant != 0 || nx1 > kMaxTileThreads) return false;
  int tj = mp->rows_per_tile;
  if (tj <= 0) {
    tj = 1;
    for (int t = nx2; t >= 1; --t)
      if (nx2 % t == 0 && t * nx1 <= 128) { tj = t; break; }
  }
  if (nx2 % tj != 0 || tj * nx1 > kMaxTileThreads) return false;
  cf.tj = tj;
  cf.chunk = mp->chunk > 0 ? mp->chunk : 2048;
  if (cf.chunk < 64 || cf.chunk > 8192 || (cf.chunk & 3)) return false;
  cf.tpp = nx2 / tj;
  // every tile form must fit the 227 KiB of shared memory a CTA can have (less the barrier)
  if (tile_smem(ms.three_d, tj, nx1, cf.chunk) > 227 * 1024 - 256) return false;
  return true;
}

template <int MODE, int D3, int SCHEME>
int launch_tile_d(const Geo &G, const Cfg &cf, const PBuf &cur, const TileArgs &T, cudaStream_t st) {
  const long long tiles = (long long)G.nmb * G.nx3 * cf.tpp;
  const size_t sm = tile_smem(D3, cf.tj, G.nx1, cf.chunk);
  static size_t configured = 0;
  if (sm > 48 * 1024 && sm > configured) {
    cudaFuncSetAttribute(k_tile<MODE, D3, SCHEME>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    configured = sm;
  }
  k_tile<MODE, D3, SCHEME><<<(unsigned)tiles, cf.tj * G.nx1, sm, st>>>(cur, G, T);
  return dustb_host::launch_status("mixed tile");
}

template <int MODE>
int launch_tile(const MState &S, const PBuf &cur, const Geo &G, const Cfg &cf, TileArgs T,
                cudaStream_t st) {
  T.tj = cf.tj; T.chunk = cf.chunk; T.tpp = cf.tpp; T.cstart = S.cstart;
  // one kernel per dimensionality and deposit scheme (no per-particle scheme selection)
  if (G.three_d) {
    if (G.scheme == 2) return launch_tile_d<MODE, 1, 2>(G, cf, cur, T, st);
    if (G.scheme == 1) return launch_tile_d<MODE, 1, 1>(G, cf, cur, T, st);
    return launch_tile_d<MODE, 1, 0>(G, cf, cur, T, st);
  }
  if (G.scheme == 2) return launch_tile_d<MODE, 0, 2>(G, cf, cur, T, st);
  if (G.scheme == 1) return launch_tile_d<MODE, 0, 1>(G, cf, cur, T, st);
  return launch_tile_d<MODE, 0, 0>(G, cf, cur, T, st);
}

// sort copy src into dst by the cells it holds (histogram, scan, moves)
int sort_into(const MState &S, const PBuf &src, const PBuf &dst, const dustb_mesh &ms, int n,
              cudaStream_t st) {
  const long long ncell = ncell_of(ms);
  cudaMemsetAsync(S.cstart, 0, 4 * (size_t)(ncell + 1), st);
  if (n > 0) k_hist<<<nblk(n), kT, 0, st>>>(src.cell, n, S.cstart);
  int rc = exclusive_scan(S.cstart, ncell + 1, S.bsum, st);
  if (rc) return rc;
  cudaMemcpyAsync(S.cursor, S.cstart, 4 * (size_t)(ncell + 1), cudaMemcpyDeviceToDevice, st);
  if (n > 0) k_sortmove<<<nblk(n), kT, 0, st>>>(src, dst, n, S.cursor);
  return dustb_host::launch_status("mixed sort");
}

bool params_ok(const dustb_ctx *c, const dustb_mixed_params *mp) {
  if (!dustb_cells::ctx_valid(c) || !mp) return false;
  for (int a = 0; a < 3; ++a)
    if (!(mp->dx[a] > 0.0)) return false;
  if (ncell_of(c->mesh) >= (1LL << 31)) return false;
  return true;
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
  if (!params_ok(c, mp)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  Geo G = make_geo(c, mp);
  const int n = c->part.npart;
  const long long ncell = ncell_of(c->mesh);
  cudaMemsetAsync(S.head, 0, sizeof(MHead), st);   // the rows carry every kick so far
  cudaMemsetAsync(S.cstart, 0, 4 * (size_t)(ncell + 1), st);
  if (n > 0)
    k_import<<<nblk(n), kT, 0, st>>>(c->part.pr, c->part.pi, c->part.stride, n, S.B, S.cstart, G, c->err);
  int rc = exclusive_scan(S.cstart, ncell + 1, S.bsum, st);
  if (rc) return rc;
  cudaMemcpyAsync(S.cursor, S.cstart, 4 * (size_t)(ncell + 1), cudaMemcpyDeviceToDevice, st);
  if (n > 0) k_sortmove<<<nblk(n), kT, 0, st>>>(S.B, S.A, n, S.cursor);
  return dustb_host::launch_status("mixed_import");
}

int dustb_mixed_export(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws,
                       long long bytes, void *stream) {
  if (!params_ok(c, mp)) return DUSTB_EINVAL;
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
  if (co->sh[0] != 0.0 || co->sh[1] != 0.0) return DUSTB_EUNSUP;   // shear shift: FP64 form
  if (c->mesh.x3bc != DUSTB_X3_PERIODIC) return DUSTB_EUNSUP;       // physical x3: FP64 form
  if (!c->mesh.multi_d) return DUSTB_EUNSUP;                        // 1-D: FP64 form
  if (c->mesh.shear_x1) return DUSTB_EUNSUP;                        // shearing box: FP64 form
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  Cfg cf;
  if (!pick_cfg(c->mesh, mp, cf)) return DUSTB_EUNSUP;
  cudaStream_t st = (cudaStream_t)stream;
  Geo G = make_geo(c, mp);
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
      if (stage == 2 && br) dustb_cells::history(c, atw22 * dt, st);
    }
    PushArgs P;
    P.gam0 = (float)gam0[stage - 1]; P.gam1 = (float)gam1[stage - 1];
    P.atw_dt = (stage == 2) ? (float)(atw22 * dt) : 0.0f;
    P.bdt = (float)(beta[stage - 1] * dt);
    for (int a = 0; a < 3; ++a) P.bdx[a] = (float)(beta[stage - 1] * dt * G.inv_dx[a]);
    P.a_dt = a_dt; P.stage2 = (stage == 2);
    P.sbox = c->phys.shearing_box; P.strat = c->phys.stratified;
    P.q = (float)c->phys.qshear; P.om = (float)c->phys.omega0;
    // stage 2: stage 1's consistent kick (this cycle's split); stage 1: the previous
    // cycle's stage-2 kick, if it left one pending
    P.res = (stage == 1 || (br && cons)) ? c->f.resid : nullptr;
    P.head = S.head;
    P.set_pending = (stage == 2 && br && cons);
    P.err = c->err;
    {
      Scope sc(DUSTB_K_PUSH, st);
      cudaMemsetAsync(S.cstart, 0, 4 * (size_t)(ncell + 1), st);
      if (n > 0) k_count<<<nblk(n), kT, 0, st>>>(src, S.key, S.cstart, G, n, P);
      RUN(dustb_host::launch_status("mixed count"));
    }
    {
      Scope sc(DUSTB_K_FILL, st);
      RUN(exclusive_scan(S.cstart, ncell + 1, S.bsum, st));
      cudaMemcpyAsync(S.cursor, S.cstart, 4 * (size_t)(ncell + 1), cudaMemcpyDeviceToDevice, st);
    }
    {
      Scope sc(DUSTB_K_PUSH, st);
      if (n > 0) k_move<<<nblk(n), kT, 0, st>>>(src, cur, S.key, S.cursor, G, n, P);
      RUN(dustb_host::launch_status("mixed move"));
      if (stage == 1) cudaMemsetAsync(&S.head->pending, 0, sizeof(int), st);   // applied
    }
    TileArgs T{};
    T.a_dt = a_dt; T.err = c->err; T.deposit = 1;
    if (br) {
      Scope sc(DUSTB_K_DEPOSIT_QP, st);
      cudaMemsetAsync(c->f.qdep, 0, fbytes * 5, st);
      T.dfield = c->f.qdep; T.dnvar = 5; T.res = c->f.resid;
      RUN(launch_tile<MODE_QP>(S, cur, G, cf, T, st));
    }
    // the deposits go straight into the owners' active cells and the gathers read ghost
    // cells from their owners, so no ghost exchange of qdep, work, dmom or u* is needed
    {
      Scope sc(DUSTB_K_CELLS, st);
      RUN(dustb_solve_ustar(c, st));
    }
    if (br && c->phys.drag_solver >= DUSTB_SOLVER_DC1) {
      const int nsw = (c->phys.drag_solver == DUSTB_SOLVER_DC2) ? 2 : 1;
      for (int w = 0; w < nsw; ++w) {
        cudaMemsetAsync(c->f.work, 0, fbytes * 3, st);
        { Scope sc(DUSTB_K_OPERATOR, st);
          T.gfield = c->f.ustar; T.dfield = c->f.work; T.dnvar = 3;
          RUN(launch_tile<MODE_OP>(S, cur, G, cf, T, st)); }
        { Scope sc(DUSTB_K_CELLS, st);
          dustb_cells::dc_correct(c, st); }
      }
    }
    if (br) cudaMemsetAsync(c->f.dmom, 0, fbytes * 3, st);
    {
      Scope sc(DUSTB_K_KICK, st);
      T.gfield = c->f.ustar; T.dfield = c->f.dmom; T.dnvar = 3; T.deposit = br;
      RUN(launch_tile<MODE_KICK>(S, cur, G, cf, T, st));
    }
    if (br) {
      { Scope sc(DUSTB_K_CELLS, st);
        if (cons) dustb_cells::consistent_gas(c, a_dt, st);
        else dustb_cells::pmbr(c, a_dt, st); }
      // stage 2's consistent dust kick is left pending (recorded by stage 2's count): the
      // next cycle's stage-1 push, or an export, applies it
    }
  }
  {
    // the gas tail's ghost exchange of the conserved state, once per cycle (nothing in the
    // drag step reads u0's ghost cells between the stages)
    Scope sc(DUSTB_K_CELLS, st);
    RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, st));
  }
#undef RUN
  return DUSTB_OK;
}

}  // extern "C"
