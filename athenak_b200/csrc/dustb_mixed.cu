// dustb_mixed.cu -- the mixed-precision form of the imex2+ drag step.
//
// Particle shadow (structure of arrays, 4-byte words): packed cell id (block, k, j, i),
// FP32 offsets inside the cell, velocity, velocity register, register displacement x1 - x
// in cells, drag rate, stopping time, mass, and the particle's row in the reference SoA.
// The mesh fields are the reference's FP64 arrays.
//
// One stage (the task order of src/dust/dust_tasks.cpp:56-107):
//   push      per particle: [stage 2: the stage-1 consistent dust kick], register copy,
//             the explicit push, the cell/block carry that replaces SetNewPrtclGID, and the
//             per-cell histogram of the new cells
//   csr       scan of the histogram and the cell -> particles order (dustb_sort.cu)
//   deposit   per CTA a tile of rows of cells; every thread owns one source cell and one z
//             offset, sums the 9 (y, x) stencil weights times the deposited values of its
//             cell's particles in registers, adds them into an FP64 shared-memory window in 9
//             conflict-free passes, and the window is added to the FP64 field once per cell
//             (global FP64 atomics only across tile borders).  Three forms: Q/P + centre mass
//             (DepositDrag), the dc1 operator gather/deposit (PointOperatorParticles) and
//             the gather-kick-deposit (GatherKickPMBR), the gathers reading an FP32 copy of the
//             tile's u* window from shared memory.
//   cells     the FP64 per-cell solves and exchanges of dustb_fp64.cu
//   kick      [stage 2] the consistent dust kick (stage 1's is folded into stage 2's push)
// Weights, gathers and kicks are FP32; the drag factor a/(t_s + a) is formed in FP64; every
// deposit is accumulated into FP64.  The kick deposits the velocity change the particle
// actually received (v_new - v in FP32), so gas + dust momentum is conserved to the FP64
// round-off of the accumulation.
#include <cfloat>
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
constexpr int kMaxTileThreads = 384;
constexpr int kNFloat = 18;

inline unsigned nblk(long long n) {
  long long b = (n + kT - 1) / kT;
  return (unsigned)(b < 1 ? 1 : b);
}
inline size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

struct MState {
  int *cell, *order, *pid;
  float *ox, *oy, *oz, *vx, *vy, *vz, *ax, *ay, *az, *wx, *wy, *wz, *rx, *ry, *rz, *ts, *m;
  float *cc;                   // drag factor a/(t_s + a) of the cycle (formed in FP64)
  float *tmp;
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

// every FP32 particle array of the shadow, in one place (carving and permuting use it)
inline void float_arrays(MState &S, float **fp[kNFloat]) {
  float **all[kNFloat] = {&S.ox, &S.oy, &S.oz, &S.vx, &S.vy, &S.vz, &S.ax, &S.ay, &S.az,
                          &S.wx, &S.wy, &S.wz, &S.rx, &S.ry, &S.rz, &S.ts, &S.m, &S.cc};
  static_assert(sizeof(all) / sizeof(all[0]) == kNFloat, "shadow array list");
  for (int f = 0; f < kNFloat; ++f) fp[f] = all[f];
}

long long ncell_of(const dustb_mesh &ms) {
  return (long long)ms.nmb * ms.nx1 * (ms.multi_d ? ms.nx2 : 1) * (ms.three_d ? ms.nx3 : 1);
}

// workspace carving (the same order in every call)
bool carve(const dustb_mesh &ms, int n, void *ws, long long bytes, MState &S, long long *need) {
  const long long ncell = ncell_of(ms);
  size_t N = (size_t)(n > 0 ? n : 1);
  size_t off = 0;
  size_t o_cell = off; off += al256(4 * N);
  size_t o_order = off; off += al256(4 * N);
  size_t o_pid = off; off += al256(4 * N);
  size_t o_f[kNFloat];
  for (int f = 0; f < kNFloat; ++f) { o_f[f] = off; off += al256(4 * N); }
  size_t o_tmp = off; off += al256(4 * N);
  size_t o_cs = off; off += al256(4 * (size_t)(ncell + 1));
  size_t o_cur = off; off += al256(4 * (size_t)(ncell + 1));
  size_t o_bs = off; off += al256(4 * (size_t)scan_bsum_ints(ncell + 1));
  if (need) *need = (long long)off;
  if (!ws || bytes < (long long)off) return false;
  char *b = (char *)ws;
  S.cell = (int *)(b + o_cell); S.order = (int *)(b + o_order); S.pid = (int *)(b + o_pid);
  float **fp[kNFloat];
  float_arrays(S, fp);
  for (int f = 0; f < kNFloat; ++f) *fp[f] = (float *)(b + o_f[f]);
  S.tmp = (float *)(b + o_tmp);
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

__device__ __forceinline__ void warp_hist(int *count, int key, bool live) {
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  const unsigned peers = __match_any_sync(act, key);
  const int lane = threadIdx.x & 31;
  if (lane == __ffs(peers) - 1) atomicAdd(&count[key], __popc(peers));
}

// ---- import / export ------------------------------------------------------------------
__global__ void k_import(const double *pr, const int *pi, long long stride, int n, MState S,
                         Geo G, unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  bool live = p < n;
  int key = 0;
  if (live) {
    auto R = [&](int r) { return pr[(long long)r * stride + p]; };
    int m = pi[(long long)DUSTB_PGID * stride + p] - G.gids;
    if (m < 0 || m >= G.nmb) { report(err, DUSTB_ERR_PGID); m = m < 0 ? 0 : G.nmb - 1; }
    const double *sz = G.mb + (long long)m * 9;
    const int nx[3] = {G.nx1, G.nx2, G.nx3};
    const double x[3] = {R(DUSTB_IPX), R(DUSTB_IPY), R(DUSTB_IPZ)};
    const double x1[3] = {R(DUSTB_IPX1), R(DUSTB_IPY1), R(DUSTB_IPZ1)};
    int ic[3];
    float of[3], dd[3];
    for (int a = 0; a < 3; ++a) {
      if (a == 2 && !G.three_d) { ic[2] = 0; of[2] = 0.5f; dd[2] = 0.0f; break; }
      double cell = (x[a] - sz[a]) * ((double)nx[a] / (sz[3 + a] - sz[a]));
      int ig = (int)(cell + 1.0) - 1;
      if (ig < 0 || ig >= nx[a]) { report(err, DUSTB_ERR_HALO); ig = ig < 0 ? 0 : nx[a] - 1; }
      double o = cell - (double)ig;
      float fo = (float)o;
      if (!(fo >= 0.0f)) fo = 0.0f;
      if (fo >= 1.0f) fo = 0.99999994f;
      ic[a] = ig; of[a] = fo;
      dd[a] = (float)((x1[a] - x[a]) * G.inv_dx[a]);
    }
    key = encode(G, m, ic[2], ic[1], ic[0]);
    S.cell[p] = key; S.pid[p] = p;
    S.ox[p] = of[0]; S.oy[p] = of[1]; S.oz[p] = of[2];
    S.vx[p] = (float)R(DUSTB_IPVX); S.vy[p] = (float)R(DUSTB_IPVY); S.vz[p] = (float)R(DUSTB_IPVZ);
    S.ax[p] = dd[0]; S.ay[p] = dd[1]; S.az[p] = dd[2];
    S.wx[p] = (float)R(DUSTB_IPVX1); S.wy[p] = (float)R(DUSTB_IPVY1); S.wz[p] = (float)R(DUSTB_IPVZ1);
    S.rx[p] = (float)R(DUSTB_IPRX); S.ry[p] = (float)R(DUSTB_IPRY); S.rz[p] = (float)R(DUSTB_IPRZ);
    S.ts[p] = (float)R(DUSTB_IPTS); S.m[p] = (float)R(DUSTB_IPM);
  }
  warp_hist(S.cstart, key, live);
}

__global__ void k_export(double *pr, int *pi, long long stride, int n, MState S, Geo G) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  int m, k, j, i;
  decode(G, S.cell[q], m, k, j, i);
  const int p = S.pid[q];
  auto W = [&](int r, double v) { pr[(long long)r * stride + p] = v; };
  const double *sz = G.mb + (long long)m * 9;
  const double x = sz[X1MIN] + ((double)i + (double)S.ox[q]) * G.dx[0];
  const double y = sz[X2MIN] + ((double)j + (double)S.oy[q]) * G.dx[1];
  W(DUSTB_IPX, x); W(DUSTB_IPY, y);
  W(DUSTB_IPX1, x + (double)S.ax[q] * G.dx[0]);
  W(DUSTB_IPY1, y + (double)S.ay[q] * G.dx[1]);
  if (G.three_d) {
    const double z = sz[X3MIN] + ((double)k + (double)S.oz[q]) * G.dx[2];
    W(DUSTB_IPZ, z);
    W(DUSTB_IPZ1, z + (double)S.az[q] * G.dx[2]);
  }
  W(DUSTB_IPVX, S.vx[q]); W(DUSTB_IPVY, S.vy[q]); W(DUSTB_IPVZ, S.vz[q]);
  W(DUSTB_IPVX1, S.wx[q]); W(DUSTB_IPVY1, S.wy[q]); W(DUSTB_IPVZ1, S.wz[q]);
  W(DUSTB_IPRX, S.rx[q]); W(DUSTB_IPRY, S.ry[q]); W(DUSTB_IPRZ, S.rz[q]);
  pi[(long long)DUSTB_PGID * stride + p] = m + G.gids;
}

// histogram of the current cells (sort)
__global__ void k_hist(const int *cell, int n, int *count) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  bool live = p < n;
  warp_hist(count, live ? cell[p] : 0, live);
}

__global__ void k_gather_i(const int *src, const int *order, int n, int *dst) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) dst[q] = src[order[q]];
}
__global__ void k_gather_f(const float *src, const int *order, int n, float *dst) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) dst[q] = src[order[q]];
}

// ---- push + carry + histogram ----------------------------------------------------------
struct PushArgs {
  float gam0, gam1, atw_dt;
  float bdt;                  // beta*dt (velocity kick)
  float bdx[3];               // beta*dt/dx per axis (drift in cells)
  double a_dt;
  int stage2;
  int sbox, strat;
  float q, om;
  const double *res;          // stage 2 with the consistent split: stage 1's dust residual
  unsigned *err;
};

__global__ void __launch_bounds__(kT) k_push(MState S, Geo G, int n, PushArgs P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  bool live = p < n;
  int key = 0;
  if (live) {
    int m, k, j, i;
    decode(G, S.cell[p], m, k, j, i);
    float ox = S.ox[p], oy = S.oy[p], oz = S.oz[p];
    float vx = S.vx[p], vy = S.vy[p], vz = S.vz[p];
    float v1x, v1y, v1z, dx1, dy1, dz1, rx, ry, rz;
    if (P.stage2) {
      v1x = S.wx[p]; v1y = S.wy[p]; v1z = S.wz[p];
      dx1 = S.ax[p]; dy1 = S.ay[p]; dz1 = S.az[p];
      rx = S.rx[p]; ry = S.ry[p]; rz = S.rz[p];
      if (P.res && S.m[p] > 0.0f) {
        // dust_imex_point_consistent_dust of stage 1 (src/dust/dust_pm.cpp:686-696)
        const double cj = (double)S.cc[p];
        const long long b = G.at(m, 4, 0, k + G.ks, j + G.js, i + G.is);
        const double d0 = cj * P.res[b], d1 = cj * P.res[b + G.vstride], d2 = cj * P.res[b + 2 * G.vstride];
        vx += (float)d0; vy += (float)d1; vz += (float)d2;
        rx += (float)(d0 / P.a_dt); ry += (float)(d1 / P.a_dt); rz += (float)(d2 / P.a_dt);
      }
    } else {
      // FirstTwoImpRK: (x1, v1) <- (x, v)
      v1x = vx; v1y = vy; v1z = vz;
      dx1 = 0.0f; dy1 = 0.0f; dz1 = 0.0f;
      rx = 0.0f; ry = 0.0f; rz = 0.0f;
      S.wx[p] = vx; S.wy[p] = vy; S.wz[p] = vz;
      // the drag factor of this cycle, a/(t_s + a) (dust_pm.cpp:255), formed in FP64 once
      S.cc[p] = (float)(P.a_dt / ((double)S.ts[p] + P.a_dt));
    }
    // ExplicitPush imex (src/dust/dust_push.cpp:262-297)
    float fx = 0.0f, fy = 0.0f, fz = 0.0f, xsh = 0.0f;
    if (P.sbox) {
      const double *sz = G.mb + (long long)m * 9;
      if (G.three_d) {
        fx = 2.0f * P.om * vy;
        fy = -(2.0f - P.q) * P.om * vx;
        if (P.strat) fz = -(P.om * P.om) * (float)(sz[X3MIN] + ((double)k + oz) * G.dx[2]);
        xsh = P.q * P.om * (float)(sz[X1MIN] + ((double)i + ox) * G.dx[0]);
      } else {
        fx = 2.0f * P.om * vz;
        fz = -(2.0f - P.q) * P.om * vx;
      }
    }
    const float nvx = P.gam0 * vx + P.gam1 * v1x + P.bdt * fx + P.atw_dt * rx;
    const float nvy = P.gam0 * vy + P.gam1 * v1y + P.bdt * fy + P.atw_dt * ry;
    const float nvz = P.gam0 * vz + P.gam1 * v1z + P.bdt * fz + P.atw_dt * rz;
    // drift in cell units: x <- x + gam1 (x1 - x) + beta dt xdot (gam0 + gam1 = 1)
    const float sx = P.gam1 * dx1 + P.bdx[0] * vx;
    const float sy = P.gam1 * dy1 + P.bdx[1] * (vy - xsh);
    ox += sx; dx1 -= sx;
    oy += sy; dy1 -= sy;
    if (G.three_d) {
      const float sz_ = P.gam1 * dz1 + P.bdx[2] * vz;
      oz += sz_; dz1 -= sz_;
    }
    // cell carry (the integer part of the new offsets)
    int ci = (int)floorf(ox); ox -= (float)ci; if (ox >= 1.0f) { ox -= 1.0f; ++ci; }
    int cj = (int)floorf(oy); oy -= (float)cj; if (oy >= 1.0f) { oy -= 1.0f; ++cj; }
    int ck = 0;
    if (G.three_d) { ck = (int)floorf(oz); oz -= (float)ck; if (oz >= 1.0f) { oz -= 1.0f; ++ck; } }
    i += ci; j += cj; k += ck;
    // block crossing: the neighbour in the crossing direction (periodic images are neighbours)
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
    key = encode(G, m, k, j, i);
    S.cell[p] = key;
    S.ox[p] = ox; S.oy[p] = oy; S.oz[p] = oz;
    S.vx[p] = nvx; S.vy[p] = nvy; S.vz[p] = nvz;
    S.ax[p] = dx1; S.ay[p] = dy1; S.az[p] = dz1;
    if (P.stage2) { S.rx[p] = rx; S.ry[p] = ry; S.rz[p] = rz; }
  }
  warp_hist(S.cstart, key, live);
}

// ---- stage-2 consistent dust kick ------------------------------------------------------
__global__ void k_consistent_kick(MState S, Geo G, int n, double a_dt, const double *res) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || !(S.m[p] > 0.0f)) return;
  int m, k, j, i;
  decode(G, S.cell[p], m, k, j, i);
  const double cj = (double)S.cc[p];
  const long long b = G.at(m, 4, 0, k + G.ks, j + G.js, i + G.is);
  const double d0 = cj * res[b], d1 = cj * res[b + G.vstride], d2 = cj * res[b + 2 * G.vstride];
  S.vx[p] += (float)d0; S.vy[p] += (float)d1; S.vz[p] += (float)d2;
  S.rx[p] += (float)(d0 / a_dt); S.ry[p] += (float)(d1 / a_dt); S.rz[p] += (float)(d2 / a_dt);
}

// ---- tile deposit kernels ---------------------------------------------------------------
enum { MODE_QP = 0, MODE_OP = 1, MODE_KICK = 2 };

struct TileArgs {
  int tj, chunk, tpp;          // rows per tile, particles per pass, tiles per (block, plane)
  double a_dt;
  const double *gfield;        // gather field (3 vars), MODE_OP / MODE_KICK
  double *dfield;              // deposit field
  int dnvar;
  double *res;                 // MODE_QP: resid, the centre mass goes to var 3
  int deposit;                 // 0: kick only (no back-reaction)
  unsigned *err;
};

__host__ __device__ inline int tile_ncomp(int mode) { return mode == MODE_QP ? 4 : 3; }

template <int MODE>
__global__ void __launch_bounds__(kMaxTileThreads, 2) k_tile(MState S, Geo G, TileArgs T) {
  constexpr int NC = (MODE == MODE_QP) ? 4 : 3;
  constexpr int B = 4;                           // particles per thread loaded together
  extern __shared__ __align__(16) unsigned char smem[];
  const int nx1 = G.nx1, tj = T.tj;
  const int nct = tj * nx1;                      // source cells of the tile
  const int WK = G.three_d ? 3 : 1;
  const int WJ = tj + 2, WI = nx1 + 2;
  const int WN = WK * WJ * WI;
  // tile coordinates
  int t = blockIdx.x;
  const int per_block = G.nx3 * T.tpp;
  const int m = t / per_block;
  t -= m * per_block;
  const int k = t / T.tpp;
  const int j0 = (t - k * T.tpp) * tj;
  const int c0 = encode(G, m, k, j0, 0);
  // shared layout: cstart | gather window (float4) | deposit window (FP64) | chunk SoA
  int *s_cs = (int *)smem;
  size_t off = ((size_t)(nct + 1) * 4 + 15) & ~(size_t)15;
  float4 *gw = (float4 *)(smem + off);
  if (MODE != MODE_QP) off += (size_t)WN * 16;
  double *dw = (double *)(smem + off);           // [NC][WN]
  off += (size_t)NC * WN * 8;
  float *s_f = (float *)(smem + off);            // [9 weights + NC values][chunk]
  const int CH = T.chunk;

  for (int x = threadIdx.x; x <= nct; x += blockDim.x) s_cs[x] = S.cstart[c0 + x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
  // threads of this warp (the last warp of a block of 8-cell rows can be partial)
  const int wlanes = min(32, (int)blockDim.x - 32 * warp);
  if (MODE != MODE_QP) {
    // the tile's u* window; cells beyond the block read the owning neighbour's active cell
    // (the same-level copy exchange of the ghost cells, folded into the load)
    for (int row = warp; row < WK * WJ; row += nwarp) {
      const int wk = row / WJ, wj = row - wk * WJ;
      for (int wi = lane; wi < WI; wi += wlanes) {
        int kk = G.three_d ? (k - 1 + wk) : 0, jj = j0 - 1 + wj, ii = wi - 1, mo;
        float4 g = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (G.owner(m, kk, jj, ii, mo)) {
          const long long b = G.at(mo, 3, 0, G.ks + kk, G.js + jj, G.is + ii);
          g = make_float4((float)T.gfield[b], (float)T.gfield[b + G.vstride],
                          (float)T.gfield[b + 2 * G.vstride], 0.0f);
        }
        gw[row * WI + wi] = g;
      }
    }
  }
  if (T.deposit)
    for (int w = threadIdx.x; w < NC * WN; w += blockDim.x) dw[w] = 0.0;
  __syncthreads();
  const int P0 = s_cs[0], P1 = s_cs[nct];
  // thread role in the accumulation: source cell cl, z offset cz
  const int cl = threadIdx.x % nct;
  const int cz = threadIdx.x / nct;              // 0..WK-1
  const int cj_l = cl / nx1, ci_l = cl - cj_l * nx1;
  float qt = 0.0f;
  const float inv_vol = (float)(1.0 / G.vol);
  const float inv_adt = (float)(1.0 / T.a_dt);

  for (int cbase = P0; cbase < P1; cbase += CH) {
    const int cnt = min(CH, P1 - cbase);
    // (a) per particle: the 9 stencil weights, [gather, kick] and the deposited values into
    // shared memory (once, for the 3 z-offset threads of the cell); the loads of B particles
    // per thread are issued together
    for (int x0 = threadIdx.x; x0 < cnt; x0 += B * blockDim.x) {
      int pb[B];
#pragma unroll
      for (int u = 0; u < B; ++u) pb[u] = S.order[cbase + min(x0 + u * (int)blockDim.x, cnt - 1)];
      int lc[B];
      float fo[B][3], fc[B], fmass[B], fv[B][3];
#pragma unroll
      for (int u = 0; u < B; ++u) {
        const int p = pb[u];
        lc[u] = S.cell[p] - c0;
        fo[u][0] = S.ox[p]; fo[u][1] = S.oy[p]; fo[u][2] = S.oz[p];
        fc[u] = S.cc[p]; fmass[u] = S.m[p];
        if (MODE != MODE_OP) { fv[u][0] = S.vx[p]; fv[u][1] = S.vy[p]; fv[u][2] = S.vz[p]; }
      }
#pragma unroll
      for (int u = 0; u < B; ++u) {
        const int x = x0 + u * blockDim.x;
        if (x >= cnt) break;
        const int local = lc[u];               // the tile's cells are consecutive ids
        if (local < 0 || local >= nct) {
          // not a particle of this tile: the cell index is stale; contribute nothing
          report(T.err, DUSTB_ERR_WINDOW);
#pragma unroll
          for (int q = 0; q < 9 + NC; ++q) s_f[q * CH + x] = 0.0f;
          continue;
        }
        int jl, pii;
        if (G.l1 >= 0) { jl = local >> G.l1; pii = local & (nx1 - 1); }
        else { jl = local / nx1; pii = local - jl * nx1; }
        const float c32 = fc[u], mass = fmass[u];
        float wx_[3], wy_[3], wz_[3];
        wts(G.scheme, fo[u][0], wx_); wts(G.scheme, fo[u][1], wy_);
        if (G.three_d) wts(G.scheme, fo[u][2], wz_); else { wz_[0] = 0.0f; wz_[1] = 1.0f; wz_[2] = 0.0f; }
        float qv[NC];
        if (MODE == MODE_QP) {
          const float mc = mass * c32 * inv_vol;
          qv[0] = mc; qv[1] = mc * fv[u][0]; qv[2] = mc * fv[u][1];
          if (NC > 3) qv[NC - 1] = mc * fv[u][2];
        } else {
          float ux = 0.0f, uy = 0.0f, uz = 0.0f;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if (!G.three_d && c != 1) continue;
            const int wk = G.three_d ? c : 0;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
              const float wzy = wz_[c] * wy_[b];
              const float4 *row = gw + (wk * WJ + jl + b) * WI + pii;
#pragma unroll
              for (int a = 0; a < 3; ++a) {
                const float w = wzy * wx_[a];
                const float4 g = row[a];
                ux = fmaf(w, g.x, ux); uy = fmaf(w, g.y, uy); uz = fmaf(w, g.z, uz);
              }
            }
          }
          if (MODE == MODE_OP) {
            const float mc = mass * c32 * inv_vol;
            qv[0] = mc * ux; qv[1] = mc * uy; qv[2] = mc * uz;
          } else {
            // GatherKickPMBR (src/dust/dust_pm.cpp:534-563) with the applied velocity change
            const float vx = fv[u][0], vy = fv[u][1], vz = fv[u][2];
            const float nx_ = vx + c32 * (ux - vx), ny_ = vy + c32 * (uy - vy), nz_ = vz + c32 * (uz - vz);
            const float dvx = nx_ - vx, dvy = ny_ - vy, dvz = nz_ - vz;
            const int p = pb[u];
            S.vx[p] = nx_; S.vy[p] = ny_; S.vz[p] = nz_;
            S.rx[p] = dvx * inv_adt; S.ry[p] = dvy * inv_adt; S.rz[p] = dvz * inv_adt;
            const float fac = -mass * inv_vol;
            qv[0] = fac * dvx; qv[1] = fac * dvy; qv[2] = fac * dvz;
          }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          s_f[a * CH + x] = wx_[a]; s_f[(3 + a) * CH + x] = wy_[a]; s_f[(6 + a) * CH + x] = wz_[a];
        }
#pragma unroll
        for (int q = 0; q < NC; ++q) s_f[(9 + q) * CH + x] = qv[q];
      }
    }
    __syncthreads();
    if (T.deposit) {
      // (b) per source cell and z offset: the 9 stencil sums of the cell's particles
      float acc[3][3][NC];
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int q = 0; q < NC; ++q) acc[b][a][q] = 0.0f;
      const int lo = max(s_cs[cl], cbase) - cbase;
      const int hi = min(s_cs[cl + 1], cbase + cnt) - cbase;
      const int zrow = (G.three_d ? 6 + cz : 7) * CH;
      for (int r = lo; r < hi; ++r) {
        const float wx_[3] = {s_f[r], s_f[CH + r], s_f[2 * CH + r]};
        const float wy_[3] = {s_f[3 * CH + r], s_f[4 * CH + r], s_f[5 * CH + r]};
        const float wzc = s_f[zrow + r];
        float qv[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) qv[q] = s_f[(9 + q) * CH + r];
        if (MODE == MODE_QP && cz == (G.three_d ? 1 : 0)) qt += qv[0];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const float wzy = wzc * wy_[b];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const float w = wzy * wx_[a];
#pragma unroll
            for (int q = 0; q < NC; ++q) acc[b][a][q] = fmaf(w, qv[q], acc[b][a][q]);
          }
        }
      }
      // (c) into the FP64 window: 9 passes, one (y, x) offset each; within a pass every
      // thread writes a different window cell
#pragma unroll
      for (int b = 0; b < 3; ++b) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int w = (cz * WJ + cj_l + b) * WI + ci_l + a;
#pragma unroll
          for (int q = 0; q < NC; ++q) dw[q * WN + w] += (double)acc[b][a][q];
          __syncthreads();
        }
      }
    }
  }
  if (MODE == MODE_QP && cz == (G.three_d ? 1 : 0)) {
    // centre mass m c / V of the cell (dust_imex_point_center_mass): only this tile's
    // particles have this cell as their centre, so it is stored, not added
    T.res[G.at(m, 4, 3, G.ks + k, G.js + j0 + cj_l, G.is + ci_l)] = (double)qt;
  }
  if (!T.deposit || P1 == P0) return;
  // (d) the window into the FP64 field; window cells beyond the block go straight into the
  // owning neighbour's active cell (the additive ghost exchange folded into the flush)
  for (int row = warp; row < NC * WK * WJ; row += nwarp) {
    const int q = row / (WK * WJ), r2 = row - q * (WK * WJ);
    const int wk = r2 / WJ, wj = r2 - wk * WJ;
    for (int wi = lane; wi < WI; wi += wlanes) {
      const double v = dw[row * WI + wi];
      if (v == 0.0) continue;
      int kk = G.three_d ? (k - 1 + wk) : 0, jj = j0 - 1 + wj, ii = wi - 1, mo;
      if (!G.owner(m, kk, jj, ii, mo)) continue;
      atomicAdd(&T.dfield[G.at(mo, T.dnvar, q, G.ks + kk, G.js + jj, G.is + ii)], v);
    }
  }
}

size_t tile_smem(int mode, int tj, int nx1, int three_d, int chunk) {
  const int nct = tj * nx1;
  const int WN = (three_d ? 3 : 1) * (tj + 2) * (nx1 + 2);
  const int NC = tile_ncomp(mode);
  size_t s = ((size_t)(nct + 1) * 4 + 15) & ~(size_t)15;
  if (mode != MODE_QP) s += (size_t)WN * 16;
  s += (size_t)NC * WN * 8;
  s += (size_t)(9 + NC) * chunk * 4;
  return s;
}

// One thread per source cell: the thread walks its cell's particles (cell order) straight
// from global memory, forms the 27 stencil weights and the deposited values of each,
// accumulates the 27 x NC sums in registers and adds them to the tile's FP64 shared window
// with shared-memory atomics (native FP64 on this GPU); the window is added to the FP64
// field once per cell.  Three barriers per tile.
template <int MODE>
__global__ void __launch_bounds__(256, 1) k_cellacc(MState S, Geo G, TileArgs T) {
  constexpr int NC = (MODE == MODE_QP) ? 4 : 3;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nx1 = G.nx1, tj = T.tj;
  const int nct = tj * nx1;                      // source cells of the tile (= threads)
  const int WK = G.three_d ? 3 : 1;
  const int WJ = tj + 2, WI = nx1 + 2;
  const int WN = WK * WJ * WI;
  int t = blockIdx.x;
  const int per_block = G.nx3 * T.tpp;
  const int m = t / per_block;
  t -= m * per_block;
  const int k = t / T.tpp;
  const int j0 = (t - k * T.tpp) * tj;
  const int c0 = encode(G, m, k, j0, 0);
  // shared layout: gather window (float4) | deposit window (FP64)
  size_t off = 0;
  float4 *gw = (float4 *)smem;
  if (MODE != MODE_QP) off += (size_t)WN * 16;
  double *dw = (double *)(smem + off);           // [NC][WN]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
  // threads of this warp (the last warp of a block of 8-cell rows can be partial)
  const int wlanes = min(32, (int)blockDim.x - 32 * warp);
  if (MODE != MODE_QP) {
    for (int row = warp; row < WK * WJ; row += nwarp) {
      const int wk = row / WJ, wj = row - wk * WJ;
      for (int wi = lane; wi < WI; wi += wlanes) {
        int kk = G.three_d ? (k - 1 + wk) : 0, jj = j0 - 1 + wj, ii = wi - 1, mo;
        float4 g = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (G.owner(m, kk, jj, ii, mo)) {
          const long long b = G.at(mo, 3, 0, G.ks + kk, G.js + jj, G.is + ii);
          g = make_float4((float)T.gfield[b], (float)T.gfield[b + G.vstride],
                          (float)T.gfield[b + 2 * G.vstride], 0.0f);
        }
        gw[row * WI + wi] = g;
      }
    }
  }
  if (T.deposit)
    for (int w = threadIdx.x; w < NC * WN; w += blockDim.x) dw[w] = 0.0;
  __syncthreads();
  const int cl = threadIdx.x;                    // the thread's source cell in the tile
  int jl, il;
  if (G.l1 >= 0) { jl = cl >> G.l1; il = cl & (nx1 - 1); }
  else { jl = cl / nx1; il = cl - jl * nx1; }
  const int lo = S.cstart[c0 + cl], hi = S.cstart[c0 + cl + 1];
  const float inv_vol = (float)(1.0 / G.vol);
  const float inv_adt = (float)(1.0 / T.a_dt);
  float acc[3][3][3][NC];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int q = 0; q < NC; ++q) acc[c][b][a][q] = 0.0f;
  float qt = 0.0f;
  for (int r = lo; r < hi; ++r) {
    const int p = S.order[r];
    const float c32 = S.cc[p], mass = S.m[p];
    float wx_[3], wy_[3], wz_[3];
    wts(G.scheme, S.ox[p], wx_);
    wts(G.scheme, S.oy[p], wy_);
    if (G.three_d) wts(G.scheme, S.oz[p], wz_); else { wz_[0] = 0.0f; wz_[1] = 1.0f; wz_[2] = 0.0f; }
    float qv[NC];
    if (MODE == MODE_QP) {
      const float mc = mass * c32 * inv_vol;
      qt += mc;
      qv[0] = mc; qv[1] = mc * S.vx[p]; qv[2] = mc * S.vy[p];
      if (NC > 3) qv[NC - 1] = mc * S.vz[p];
    } else {
      float ux = 0.0f, uy = 0.0f, uz = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!G.three_d && c != 1) continue;
        const int wk = G.three_d ? c : 0;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const float wzy = wz_[c] * wy_[b];
          const float4 *row = gw + (wk * WJ + jl + b) * WI + il;
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const float w = wzy * wx_[a];
            const float4 g = row[a];
            ux = fmaf(w, g.x, ux); uy = fmaf(w, g.y, uy); uz = fmaf(w, g.z, uz);
          }
        }
      }
      if (MODE == MODE_OP) {
        const float mc = mass * c32 * inv_vol;
        qv[0] = mc * ux; qv[1] = mc * uy; qv[2] = mc * uz;
      } else {
        // GatherKickPMBR (src/dust/dust_pm.cpp:534-563) with the applied velocity change
        const float vx = S.vx[p], vy = S.vy[p], vz = S.vz[p];
        const float nx_ = vx + c32 * (ux - vx), ny_ = vy + c32 * (uy - vy), nz_ = vz + c32 * (uz - vz);
        const float dvx = nx_ - vx, dvy = ny_ - vy, dvz = nz_ - vz;
        S.vx[p] = nx_; S.vy[p] = ny_; S.vz[p] = nz_;
        S.rx[p] = dvx * inv_adt; S.ry[p] = dvy * inv_adt; S.rz[p] = dvz * inv_adt;
        const float fac = -mass * inv_vol;
        qv[0] = fac * dvx; qv[1] = fac * dvy; qv[2] = fac * dvz;
      }
    }
    if (T.deposit) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!G.three_d && c != 1) continue;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          const float wzy = wz_[c] * wy_[b];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const float w = wzy * wx_[a];
#pragma unroll
            for (int q = 0; q < NC; ++q) acc[c][b][a][q] = fmaf(w, qv[q], acc[c][b][a][q]);
          }
        }
      }
    }
  }
  if (MODE == MODE_QP) {
    // centre mass m c / V of the cell (dust_imex_point_center_mass): only this thread's
    // particles have this cell as their centre, so it is stored, not added
    T.res[G.at(m, 4, 3, G.ks + k, G.js + j0 + jl, G.is + il)] = (double)qt;
  }
  if (!T.deposit) return;
  if (hi > lo) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (!G.three_d && c != 1) continue;
      const int wk = G.three_d ? c : 0;
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int w = (wk * WJ + jl + b) * WI + il + a;
#pragma unroll
          for (int q = 0; q < NC; ++q) atomicAdd(&dw[q * WN + w], (double)acc[c][b][a][q]);
        }
    }
  }
  __syncthreads();
  // the window into the FP64 field; window cells beyond the block go straight into the
  // owning neighbour's active cell (the additive ghost exchange folded into the flush)
  for (int row = warp; row < NC * WK * WJ; row += nwarp) {
    const int q = row / (WK * WJ), r2 = row - q * (WK * WJ);
    const int wk = r2 / WJ, wj = r2 - wk * WJ;
    for (int wi = lane; wi < WI; wi += wlanes) {
      const double v = dw[row * WI + wi];
      if (v == 0.0) continue;
      int kk = G.three_d ? (k - 1 + wk) : 0, jj = j0 - 1 + wj, ii = wi - 1, mo;
      if (!G.owner(m, kk, jj, ii, mo)) continue;
      atomicAdd(&T.dfield[G.at(mo, T.dnvar, q, G.ks + kk, G.js + jj, G.is + ii)], v);
    }
  }
}

size_t cellacc_smem(int mode, int tj, int nx1, int three_d) {
  const int WN = (three_d ? 3 : 1) * (tj + 2) * (nx1 + 2);
  size_t s = 0;
  if (mode != MODE_QP) s += (size_t)WN * 16;
  s += (size_t)tile_ncomp(mode) * WN * 8;
  return s;
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
  int tj, chunk, tpp, variant;
};

bool pick_cfg(const dustb_mesh &ms, const dustb_mixed_params *mp, Cfg &cf) {
  const int nx1 = ms.nx1, nx2 = ms.multi_d ? ms.nx2 : 1;
  const int wk = ms.three_d ? 3 : 1;
  cf.variant = mp->variant;
  int tj = mp->rows_per_tile;
  if (cf.variant == 0) {
    // one thread per source cell: tiles of up to 256 cells
    if (tj <= 0) {
      tj = 1;
      for (int t = nx2; t >= 1; --t)
        if (nx2 % t == 0 && t * nx1 <= 256) { tj = t; break; }
    }
    if (nx2 % tj != 0 || tj * nx1 > 256) return false;
  } else {
    if (tj <= 0) {
      tj = 1;
      for (int t = nx2; t >= 1; --t)
        if (nx2 % t == 0 && wk * t * nx1 <= 384 && t * nx1 <= 128 * (ms.three_d ? 1 : 3)) { tj = t; break; }
    }
    if (nx2 % tj != 0 || wk * tj * nx1 > kMaxTileThreads) return false;
  }
  cf.tj = tj;
  cf.chunk = mp->chunk > 0 ? mp->chunk : 1024;
  if (cf.chunk > 2048) return false;
  cf.tpp = nx2 / tj;
  return true;
}

template <int MODE>
int launch_tile(const MState &S, const Geo &G, const Cfg &cf, TileArgs T, cudaStream_t st) {
  T.tj = cf.tj; T.chunk = cf.chunk; T.tpp = cf.tpp;
  const long long tiles = (long long)G.nmb * G.nx3 * cf.tpp;
  if (cf.variant == 0) {
    const size_t sm = cellacc_smem(MODE, cf.tj, G.nx1, G.three_d);
    static size_t configured0 = 0;
    if (sm > 48 * 1024 && sm > configured0) {
      cudaFuncSetAttribute(k_cellacc<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      configured0 = sm;
    }
    k_cellacc<MODE><<<(unsigned)tiles, cf.tj * G.nx1, sm, st>>>(S, G, T);
    return dustb_host::launch_status("mixed cell tile");
  }
  const size_t sm = tile_smem(MODE, cf.tj, G.nx1, G.three_d, cf.chunk);
  static size_t configured = 0;
  if (sm > 48 * 1024 && sm > configured) {
    cudaFuncSetAttribute(k_tile<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    configured = sm;
  }
  const int threads = (G.three_d ? 3 : 1) * cf.tj * G.nx1;
  k_tile<MODE><<<(unsigned)tiles, threads, sm, st>>>(S, G, T);
  return dustb_host::launch_status("mixed tile");
}

int build_csr(const MState &S, const dustb_mesh &ms, int n, cudaStream_t st) {
  return csr_build(S.cell, n, ncell_of(ms), S.cstart, S.order, S.cursor, S.bsum, true, st);
}

int permute(const MState &S, int n, cudaStream_t st) {
  if (n <= 0) return DUSTB_OK;
  int *ti = (int *)S.tmp;
  k_gather_i<<<nblk(n), kT, 0, st>>>(S.cell, S.order, n, ti);
  cudaMemcpyAsync(S.cell, ti, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st);
  k_gather_i<<<nblk(n), kT, 0, st>>>(S.pid, S.order, n, ti);
  cudaMemcpyAsync(S.pid, ti, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st);
  MState T = S;
  float **fp[kNFloat];
  float_arrays(T, fp);
  float *fs[kNFloat];
  for (int f = 0; f < kNFloat; ++f) {
    fs[f] = *fp[f];
    if (!fs[f]) return DUSTB_EINVAL;
  }
  for (int f = 0; f < kNFloat; ++f) {
    k_gather_f<<<nblk(n), kT, 0, st>>>(fs[f], S.order, n, S.tmp);
    cudaMemcpyAsync(fs[f], S.tmp, 4 * (size_t)n, cudaMemcpyDeviceToDevice, st);
  }
  return dustb_host::launch_status("mixed permute");
}

// sort the shadow by cell: histogram, CSR, permutation
int sort_shadow(const MState &S, const dustb_mesh &ms, int n, cudaStream_t st) {
  const long long ncell = ncell_of(ms);
  cudaMemsetAsync(S.cstart, 0, 4 * (size_t)(ncell + 1), st);
  if (n > 0) k_hist<<<nblk(n), kT, 0, st>>>(S.cell, n, S.cstart);
  int rc = build_csr(S, ms, n, st);
  if (rc) return rc;
  return permute(S, n, st);
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
  cudaMemsetAsync(S.cstart, 0, 4 * (size_t)(ncell_of(c->mesh) + 1), st);
  if (n > 0) k_import<<<nblk(n), kT, 0, st>>>(c->part.pr, c->part.pi, c->part.stride, n, S, G, c->err);
  int rc = build_csr(S, c->mesh, n, st);
  if (rc) return rc;
  return permute(S, n, st);
}

int dustb_mixed_export(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws,
                       long long bytes, void *stream) {
  if (!params_ok(c, mp)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  Geo G = make_geo(c, mp);
  const int n = c->part.npart;
  if (n > 0)
    k_export<<<nblk(n), kT, 0, (cudaStream_t)stream>>>(c->part.pr, c->part.pi, c->part.stride, n, S, G);
  return dustb_host::launch_status("mixed_export");
}

int dustb_mixed_sort(const dustb_ctx *c, const dustb_mixed_params *mp, void *ws, long long bytes,
                     void *stream) {
  if (!params_ok(c, mp)) return DUSTB_EINVAL;
  MState S;
  if (!carve(c->mesh, c->part.npart, ws, bytes, S, nullptr)) return DUSTB_ESCRATCH;
  return sort_shadow(S, c->mesh, c->part.npart, (cudaStream_t)stream);
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
    {
      Scope sc(DUSTB_K_CELLS, st);
      if (stage == 1) cudaMemcpyAsync(c->f.u1, c->f.u0, fbytes * c->f.nvar_gas, cudaMemcpyDeviceToDevice, st);
      dustb_cells::gas_rk(c, gam0[stage - 1], gam1[stage - 1], st);
      if (stage == 2 && br) dustb_cells::history(c, atw22 * dt, st);
      cudaMemsetAsync(S.cstart, 0, 4 * (size_t)(ncell + 1), st);
    }
    {
      Scope sc(DUSTB_K_PUSH, st);
      PushArgs P;
      P.gam0 = (float)gam0[stage - 1]; P.gam1 = (float)gam1[stage - 1];
      P.atw_dt = (stage == 2) ? (float)(atw22 * dt) : 0.0f;
      P.bdt = (float)(beta[stage - 1] * dt);
      for (int a = 0; a < 3; ++a) P.bdx[a] = (float)(beta[stage - 1] * dt * G.inv_dx[a]);
      P.a_dt = a_dt; P.stage2 = (stage == 2);
      P.sbox = c->phys.shearing_box; P.strat = c->phys.stratified;
      P.q = (float)c->phys.qshear; P.om = (float)c->phys.omega0;
      P.res = (stage == 2 && br && cons) ? c->f.resid : nullptr;
      P.err = c->err;
      if (n > 0) k_push<<<nblk(n), kT, 0, st>>>(S, G, n, P);
      RUN(dustb_host::launch_status("mixed push"));
    }
    {
      Scope sc(DUSTB_K_FILL, st);
      RUN(build_csr(S, c->mesh, n, st));
    }
    TileArgs T{};
    T.a_dt = a_dt; T.err = c->err; T.deposit = 1;
    if (br) {
      Scope sc(DUSTB_K_DEPOSIT_QP, st);
      cudaMemsetAsync(c->f.qdep, 0, fbytes * 5, st);
      T.dfield = c->f.qdep; T.dnvar = 5; T.res = c->f.resid;
      RUN(launch_tile<MODE_QP>(S, G, cf, T, st));
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
          RUN(launch_tile<MODE_OP>(S, G, cf, T, st)); }
        { Scope sc(DUSTB_K_CELLS, st);
          dustb_cells::dc_correct(c, st); }
      }
    }
    if (br) cudaMemsetAsync(c->f.dmom, 0, fbytes * 3, st);
    {
      Scope sc(DUSTB_K_KICK, st);
      T.gfield = c->f.ustar; T.dfield = c->f.dmom; T.dnvar = 3; T.deposit = br;
      RUN(launch_tile<MODE_KICK>(S, G, cf, T, st));
    }
    if (br) {
      { Scope sc(DUSTB_K_CELLS, st);
        if (cons) dustb_cells::consistent_gas(c, a_dt, st);
        else dustb_cells::pmbr(c, a_dt, st); }
      if (cons && stage == 2 && n > 0) {
        Scope sc(DUSTB_K_CONSISTENT, st);
        k_consistent_kick<<<nblk(n), kT, 0, st>>>(S, G, n, a_dt, c->f.resid);
        RUN(dustb_host::launch_status("mixed consistent kick"));
      }
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
