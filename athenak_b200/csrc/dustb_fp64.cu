// dustb_fp64.cu -- the FP64 form of the dust drag step: one kernel per reference kernel,
// one thread per particle or per cell, FP64 global atomics for the deposits.  This is the
// straightforward GPU form of the reference's Kokkos kernels (the "plain FP64" baseline of
// the mixed-precision form in dustb_mixed.cu).  Compiled with --fmad=false so that the
// per-particle arithmetic rounds exactly as the CPU oracle's does.
#include <cfloat>
#include <cstdio>
#include <cstring>

#include "dustb_common.cuh"
#include "dustb_sort.cuh"

using namespace dustb;

namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  return (unsigned)(b < 1 ? 1 : b);
}
inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

struct PCtx {            // particle view passed by value into kernels
  double *pr;
  int *pi;
  long long stride;
  int npart;
  __device__ double &r(int c, int p) const { return pr[(long long)c * stride + p]; }
  __device__ int &i(int c, int p) const { return pi[(long long)c * stride + p]; }
};

// the refinable clouds' leaf traversal on a refined mesh (dustb_leaf_tables); on = 0: none
struct LTab {
  int on, nlev, nmb, x3per;
  int nf[3];
  double rdx[3], irdx[3], fdx[3];
  const int *fbox, *blev, *nnb, *nb, *nbs, *nbmax, *safe, *locblk;
  const long long *lockey;
};

struct MCtx {            // mesh view
  const double *mb;
  const int *nghbr;
  int gids, scheme, three_d, multi_d;
  double x1min, x1max, x2min, x2max, x3min, x3max;
  const int *blev, *nml;   // refined meshes: block levels and the 56 neighbour slots (or NULL)
  LTab lt;
  __device__ double s(int m, int f) const { return mb[(long long)m * 9 + f]; }
};

PCtx pview(const dustb_ctx *c) {
  return PCtx{c->part.pr, c->part.pi, c->part.stride, c->part.npart};
}
MCtx mview(const dustb_ctx *c) {
  const dustb_mesh &ms = c->mesh;
  MCtx M{ms.mb_size, ms.nghbr, ms.gids, c->phys.scheme, ms.three_d, ms.multi_d,
         ms.x1min, ms.x1max, ms.x2min, ms.x2max, ms.x3min, ms.x3max, ms.mb_lev,
         ms.nghbr_ml, LTab{}};
  if (const dustb_leaf_tables *t = ms.leaf) {
    LTab &L = M.lt;
    L.on = 1; L.nlev = t->nlev; L.nmb = ms.nmb; L.x3per = ms.x3bc == DUSTB_X3_PERIODIC;
    for (int a = 0; a < 3; ++a) {
      L.nf[a] = t->nfine[a];
      L.rdx[a] = t->root_dx[a];
      L.irdx[a] = 1.0 / t->root_dx[a];
      L.fdx[a] = t->root_dx[a] / (double)(1 << t->nlev);
    }
    L.fbox = t->fbox; L.blev = t->blev; L.nnb = t->nnb; L.nb = t->nb; L.nbs = t->nbs;
    L.nbmax = t->nbmax; L.safe = t->safe; L.locblk = t->locblk; L.lockey = t->lockey;
  }
  return M;
}

__device__ __forceinline__ void weights3(const MCtx &M, const Ind &d, int m, double x,
                                         double y, double z, int &ip, int &jp, int &kp,
                                         double wx[3], double wy[3], double wz[3]) {
  pm_weights(x, M.s(m, X1MIN), M.s(m, X1MAX), d.nx1, d.is, M.scheme, ip, wx);
  pm_weights(y, M.s(m, X2MIN), M.s(m, X2MAX), d.nx2, d.js, M.scheme, jp, wy);
  if (d.three_d) {
    pm_weights(z, M.s(m, X3MIN), M.s(m, X3MAX), d.nx3, d.ks, M.scheme, kp, wz);
  } else {
    kp = d.ks; wz[0] = 0.0; wz[1] = 1.0; wz[2] = 0.0;
  }
}

__device__ __forceinline__ bool halo_ok(const Ind &d, int ip, int jp, int kp) {
  if (ip < d.is - 1 || ip > d.is + d.nx1) return false;
  if (jp < d.js - 1 || jp > d.js + d.nx2) return false;
  if (d.three_d && (kp < d.ks - 1 || kp > d.ks + d.nx3)) return false;
  return true;
}

__device__ __forceinline__ double cell_vol(const MCtx &M, const Ind &d, int m) {
  double v = M.s(m, DX1) * M.s(m, DX2);
  if (d.three_d) v *= M.s(m, DX3);
  return v;
}

__device__ __forceinline__ bool block_ok(const Ind &d, int m) { return m >= 0 && m < d.nmb; }

// ---- register copy / gas stand-in / history ------------------------------------------
__global__ void k_reg_copy(PCtx P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  P.r(DUSTB_IPX1, p) = P.r(DUSTB_IPX, p);
  P.r(DUSTB_IPVX1, p) = P.r(DUSTB_IPVX, p);
  P.r(DUSTB_IPY1, p) = P.r(DUSTB_IPY, p);
  P.r(DUSTB_IPVY1, p) = P.r(DUSTB_IPVY, p);
  P.r(DUSTB_IPZ1, p) = P.r(DUSTB_IPZ, p);
  P.r(DUSTB_IPVZ1, p) = P.r(DUSTB_IPVZ, p);
}

// active-cell loop helper: idx over nmb*nx3*nx2*nx1
__device__ __forceinline__ bool active_cell(const Ind &d, long long idx, int &m, int &k, int &j,
                                            int &i) {
  long long n = (long long)d.nmb * d.nx3 * d.nx2 * d.nx1;
  if (idx >= n) return false;
  i = (int)(idx % d.nx1) + d.is; idx /= d.nx1;
  j = (int)(idx % d.nx2) + d.js; idx /= d.nx2;
  k = (int)(idx % d.nx3) + d.ks; idx /= d.nx3;
  m = (int)idx;
  return true;
}

__global__ void k_gas_rk(Ind d, double *u0, const double *u1, int nv, double g0, double g1) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  for (int v = 0; v < nv; ++v) {
    long long a = d.at(m, nv, v, k, j, i);
    u0[a] = g0 * u0[a] + g1 * u1[a];
  }
}

// (f2: a second 3-variable rate field added after dmom, in the same pass; null: none)
__global__ void k_history(Ind d, double *u0, int nv, const double *dmom, const double *f2,
                          double atw_dt) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  for (int v = 0; v < 3; ++v) {
    const long long a = d.at(m, nv, 1 + v, k, j, i), b = d.at(m, 3, v, k, j, i);
    double u = u0[a] + atw_dt * dmom[b];
    if (f2) u = u + atw_dt * f2[b];
    u0[a] = u;
  }
}

// ---- ExplicitPush imex, src/dust/dust_push.cpp:262-297 ----------------------------------
__global__ void k_push_imex(PCtx P, int three_d, int sbox, int strat, double q, double om,
                            double gam0, double gam1, double beta_dt, double atw_dt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  double x_old = P.r(DUSTB_IPX, p), y_old = P.r(DUSTB_IPY, p), z_old = P.r(DUSTB_IPZ, p);
  double vx_old = P.r(DUSTB_IPVX, p), vy_old = P.r(DUSTB_IPVY, p), vz_old = P.r(DUSTB_IPVZ, p);
  double fx = 0.0, fy = 0.0, fz = 0.0;
  if (sbox) {
    if (three_d) {
      fx = 2.0 * om * vy_old;
      fy = -(2.0 - q) * om * vx_old;
      if (strat) fz = -(om * om) * z_old;
    } else {
      fx = 2.0 * om * vz_old;
      fz = -(2.0 - q) * om * vx_old;
    }
  }
  P.r(DUSTB_IPVX, p) = gam0 * vx_old + gam1 * P.r(DUSTB_IPVX1, p) + beta_dt * fx + atw_dt * P.r(DUSTB_IPRX, p);
  P.r(DUSTB_IPVY, p) = gam0 * vy_old + gam1 * P.r(DUSTB_IPVY1, p) + beta_dt * fy + atw_dt * P.r(DUSTB_IPRY, p);
  P.r(DUSTB_IPVZ, p) = gam0 * vz_old + gam1 * P.r(DUSTB_IPVZ1, p) + beta_dt * fz + atw_dt * P.r(DUSTB_IPRZ, p);
  double ydot = vy_old;
  if (sbox && three_d) ydot -= q * om * x_old;
  P.r(DUSTB_IPX, p) = gam0 * x_old + gam1 * P.r(DUSTB_IPX1, p) + beta_dt * vx_old;
  P.r(DUSTB_IPY, p) = gam0 * y_old + gam1 * P.r(DUSTB_IPY1, p) + beta_dt * ydot;
  if (three_d) P.r(DUSTB_IPZ, p) = gam0 * z_old + gam1 * P.r(DUSTB_IPZ1, p) + beta_dt * vz_old;
}

// ---- shear-periodic x1 faces (3-D shearing box) ------------------------------------------
// Offsets formed on the host as the reference forms them: the u* / gas remap uses the unfolded
// q Omega Lx t (ShearingBox::InitRecv, shearing_box_tasks.cpp:147), the particles and the
// deposit remap the folded fmod(q Omega Lx t, Ly) (bvals_part.cpp:141, bvals_dep_general.cpp:652)
struct SBox {
  const int *sb_gid, *nghbr;
  const double *mb;
  int on, nb2, nb3, gids, nmb, nx1, nx2, nx3, ng, x3bc, drop;
  double x1min, x1max, x2min, x2max, x3min, x3max;
  double yshear, ysh, shR;
  __device__ double s(int m, int f) const { return mb[(long long)m * 9 + f]; }
  // faces of block m: bit 1 inner, bit 2 outer (bvals_part.cpp:260-261)
  __device__ int faces(int m) const {
    const double lx = s(m, X1MAX) - s(m, X1MIN);
    int f = 0;
    if (s(m, X1MIN) < x1min + 0.5 * lx) f |= 1;
    if (s(m, X1MAX) > x1max - 0.5 * lx) f |= 2;
    return f;
  }
  __device__ void b23(int m, int &b2, int &b3) const {
    b2 = (int)floor((s(m, X2MIN) - x2min) / ((x2max - x2min) / nb2) + 0.5);
    b3 = (int)floor((s(m, X3MIN) - x3min) / ((x3max - x3min) / nb3) + 0.5);
  }
  __device__ int block(int f, int b3, int b2) const {
    const int g = sb_gid[((long long)f * nb3 + b3) * nb2 + b2] - gids;
    return (g >= 0 && g < nmb) ? g : -1;
  }
  // whether direction o1 from block m crosses a shear face (remapped, not exchanged plainly)
  __device__ bool crossing(int m, int o1) const {
    if (!on || o1 == 0) return false;
    const int f = faces(m);
    return (o1 < 0) ? (f & 1) : ((f & 2) != 0);
  }
  // the active cell owning active-relative cell (k, j, i) of block m (plain neighbour table)
  __device__ bool owner(int m, int &k, int &j, int &i, int &mo) const {
    const int o1 = (i < 0) ? -1 : ((i >= nx1) ? 1 : 0);
    const int o2 = (j < 0) ? -1 : ((j >= nx2) ? 1 : 0);
    const int o3 = (k < 0) ? -1 : ((k >= nx3) ? 1 : 0);
    if ((o1 | o2 | o3) == 0) { mo = m; return true; }
    const int gid = nghbr[(long long)m * 27 + dir_slot(o1, o2, o3)];
    if (gid < 0) return false;
    mo = gid - gids;
    i -= o1 * nx1; j -= o2 * nx2; k -= o3 * nx3;
    return true;
  }
};

SBox sbview(const dustb_ctx *c) {
  const dustb_mesh &ms = c->mesh;
  SBox b{};
  b.on = ms.shear_x1 && ms.three_d;
  b.sb_gid = ms.sb_gid; b.nghbr = ms.nghbr; b.mb = ms.mb_size;
  b.nb2 = ms.sb_nb2; b.nb3 = ms.sb_nb3; b.gids = ms.gids; b.nmb = ms.nmb;
  b.nx1 = ms.nx1; b.nx2 = ms.nx2; b.nx3 = ms.nx3; b.ng = ms.ng;
  b.x3bc = ms.x3bc; b.drop = c->phys.x3_deposit_drop;
  b.x1min = ms.x1min; b.x1max = ms.x1max; b.x2min = ms.x2min; b.x2max = ms.x2max;
  b.x3min = ms.x3min; b.x3max = ms.x3max;
  if (b.on) {
    const double lx = ms.x1max - ms.x1min, ly = ms.x2max - ms.x2min;
    b.yshear = (c->phys.qshear * c->phys.omega0) * lx * ms.time;
    b.ysh = fmod(c->phys.qshear * c->phys.omega0 * lx * ms.time, ly);
    const long long N2 = (long long)ms.sb_nb2 * ms.nx2;
    b.shR = b.ysh * (double)N2 / ly;
  }
  return b;
}

// PLM_RemapFlx and a - (flx(j+1) - flx(j)) of ShearingBoxCC::PackAndSend at one row, from
// g[t] = the row's column at rows r - 2 + t (src/shearing_box/remap_fluxes.hpp:30-55)
__device__ double sb_remap(const double g[5], double eps) {
  double f[2];
  for (int h = 0; h < 2; ++h) {
    const int q = 2 + h;
    double dql, dqr;
    if (eps > 0.0) { dql = g[q - 1] - g[q - 2]; dqr = g[q] - g[q - 1]; }
    else { dql = g[q] - g[q - 1]; dqr = g[q + 1] - g[q]; }
    const double dq2 = dql * dqr;
    double dqm = 2.0 * dq2 / (dql + dqr);
    if (dq2 <= 0.0) dqm = 0.0;
    f[h] = (eps > 0.0) ? eps * (g[q - 1] + 0.5 * (1.0 - eps) * dqm)
                       : eps * (g[q] - 0.5 * (1.0 + eps) * dqm);
  }
  return g[2] - (f[1] - f[0]);
}

// ShearingBoxCC::PackAndSend + RecvAndUnpack on one device (shearing_box_cc.cpp:78-197,
// shearing_box.cpp:260-330): every cell of the x1 ghost strips of the face blocks (their
// y-ghost rows and x3 ghost planes included) takes the remapped plain-periodic strip of the
// face block holding row J -/+ joffset.  The periodic strip is read from the active cells the
// plain copy takes it from, so no cell is both read and written.
__global__ void k_shear_copy(SBox B, Ind d, double *a, int nvar) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)nvar * d.n3 * d.n2 * B.ng;
  const long long tot = 2LL * B.nb3 * B.nb2 * per;
  if (idx >= tot) return;
  const int fb = (int)(idx / per);
  long long r = idx - (long long)fb * per;
  const int i = (int)(r % B.ng); r /= B.ng;
  const int j = (int)(r % d.n2); r /= d.n2;
  const int k = (int)(r % d.n3);
  const int v = (int)(r / d.n3);
  const int n = fb / (B.nb3 * B.nb2);
  const int b3 = (fb / B.nb2) % B.nb3, b2 = fb % B.nb2;
  const int T = B.block(n, b3, b2);
  if (T < 0) return;
  const double dy = B.s(T, DX2);
  const long long joffset = (long long)(B.yshear / dy);
  double eps = fmod(B.yshear, dy) / dy;
  if (n == 1) eps *= -1.0;
  const long long Ny = (long long)B.nb2 * B.nx2;
  const long long J = (long long)b2 * B.nx2 + (j - d.js);
  long long R = (n == 0) ? J - joffset : J + joffset;
  R %= Ny; if (R < 0) R += Ny;
  const int S = B.block(n, b3, (int)(R / B.nx2));
  if (S < 0) return;
  const int rr = (int)(R % B.nx2);
  const int xr = (n == 0) ? i - B.ng : B.nx1 + i;
  double g[5];
  for (int t = 0; t < 5; ++t) {
    int kk = k - d.ks, jj = rr - 2 + t, ii = xr, mo;
    if (!B.owner(S, kk, jj, ii, mo)) return;
    g[t] = a[d.at(mo, nvar, v, d.ks + kk, d.js + jj, d.is + ii)];
  }
  a[d.at(T, nvar, v, k, j, (n == 0) ? i : d.ie + 1 + i)] = sb_remap(g, eps);
}

// The shear part of the deposit remap (DepRemapPlan part 1, bvals_dep_general.cpp:99-240) for
// active cell (k, j, i) of face block m, summed in the oracle's order (faces, source planes,
// source blocks along x2, source rows, images): the ghost cells beyond the opposite x1 face,
// moved by the box length and shifted by +shR (beyond the outer face) or -shR (beyond the inner
// face) cells, weighted by their overlap with the cell
__device__ double shear_add_sum(const SBox &B, const Ind &d, const double *a, int nvar, int m,
                                int v, int k, int j, int i) {
  const int faces = B.faces(m);
  const int ng1 = B.ng - 1;
  const long long N2 = (long long)B.nb2 * B.nx2;
  int b2, b3;
  B.b23(m, b2, b3);
  const long long J = (long long)b2 * B.nx2 + (j - d.js);
  double sum = 0.0;
  for (int side = 0; side < 2; ++side) {
    if (!(faces & (side ? 2 : 1))) continue;
    const int g = side ? i - (d.ie - ng1) : i - d.is;
    if (g < 0 || g > ng1) continue;
    const int sface = side ? 0 : 1;
    const int si = side ? g : d.ie + 1 + g;
    const double sh = side ? -B.shR : B.shR;
    const long long F = (long long)floor((double)J - sh);
    for (int zc = 0; zc < 3; ++zc) {
      int sb3 = b3, sk = k;
      if (zc == 1) {
        if (k > d.ks + ng1) continue;
        if (b3 > 0 || B.x3bc == 0) { sb3 = (b3 + B.nb3 - 1) % B.nb3; sk = k + B.nx3; }
        else if (!B.drop) { sk = 2 * d.ks - 1 - k; }
        else continue;
      } else if (zc == 2) {
        if (k < d.ke - ng1) continue;
        if (b3 < B.nb3 - 1 || B.x3bc == 0) { sb3 = (b3 + 1) % B.nb3; sk = k - B.nx3; }
        else if (!B.drop) { sk = 2 * d.ke + 1 - k; }
        else continue;
      }
      const long long Fm = ((F % N2) + N2) % N2;
      const int bc = (int)(Fm / B.nx2);
      int seen[3] = {-1, -1, -1};
      for (int db = -1; db <= 1; ++db) {
        const int sb2 = ((bc + db) % B.nb2 + B.nb2) % B.nb2;
        if (sb2 == seen[0] || sb2 == seen[1]) continue;
        seen[db + 1] = sb2;
        const int S = B.block(sface, sb3, sb2);
        if (S < 0) continue;
        for (long long Yc = F - 1; Yc <= F + 1; ++Yc)
          for (int q = -2; q <= 2; ++q) {
            const long long Y = Yc + q * N2;
            const long long sj = Y - (long long)sb2 * B.nx2 + d.js;
            if (sj < 0 || sj >= d.n2) continue;
            const double ya = (double)Y + sh, yb = (double)(Y + 1) + sh;
            for (int im = -2; im <= 2; ++im) {
              const double clo = (double)(J + im * N2), chi = clo + 1.0;
              const double o = fmin(yb, chi) - fmax(ya, clo);
              if (o > 0.0) sum += o * a[d.at(S, nvar, v, sk, (int)sj, si)];
            }
          }
      }
    }
  }
  return sum;
}

// SetNewPrtclGID's neighbour on a refined mesh (ml_route_slot, dustb_common.cuh)
__device__ int route_slot_ml(const MCtx &M, int m, int ix, int iy, int iz, int fx, int fy,
                             int fz) {
  return ml_route_slot(M.nml + (long long)m * 56, M.blev, M.gids, M.blev[m], M.mb + (long long)m * 9,
                       M.x1min, M.x2min, M.x3min, ix, iy, iz, fx, fy, fz);
}

// ---- SetNewPrtclGID, src/bvals/bvals_part.cpp:159-429 (any levels with M.nml) -------------
__global__ void k_route(PCtx P, MCtx M, Ind d, int x3bc, double *x3rem, unsigned *err, SBox B) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  int m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) { report(err, DUSTB_ERR_PGID); return; }
  const double z3a = M.x3min, z3b = M.x3max;
  if (x3bc != 0 && (P.r(DUSTB_IPZ, p) < z3a || P.r(DUSTB_IPZ, p) >= z3b)) {
    const bool lo = (P.r(DUSTB_IPZ, p) < z3a);
    if (x3bc == 1) {
      const double zf = lo ? z3a : z3b;
      double z = 2.0 * zf - P.r(DUSTB_IPZ, p);
      if (z >= z3b) z = z3b - 1.0e-12 * (z3b - z3a);
      if (z < z3a) z = z3a;
      P.r(DUSTB_IPZ, p) = z;
      P.r(DUSTB_IPVZ, p) = -P.r(DUSTB_IPVZ, p);
      P.r(DUSTB_IPZ1, p) = 2.0 * zf - P.r(DUSTB_IPZ1, p);
      P.r(DUSTB_IPVZ1, p) = -P.r(DUSTB_IPVZ1, p);
    } else {
      if (x3rem) { atomicAdd(&x3rem[0], P.r(DUSTB_IPM, p)); atomicAdd(&x3rem[1], 1.0); }
      P.r(DUSTB_IPM, p) = 0.0;
      const double dz = M.s(m, DX3);
      const double z = lo ? (M.s(m, X3MIN) + 0.5 * dz) : (M.s(m, X3MAX) - 0.5 * dz);
      P.r(DUSTB_IPZ, p) = z;
      P.r(DUSTB_IPVX, p) = 0.0; P.r(DUSTB_IPVY, p) = 0.0; P.r(DUSTB_IPVZ, p) = 0.0;
      P.r(DUSTB_IPX1, p) = P.r(DUSTB_IPX, p); P.r(DUSTB_IPY1, p) = P.r(DUSTB_IPY, p);
      P.r(DUSTB_IPZ1, p) = z;
      P.r(DUSTB_IPVX1, p) = 0.0; P.r(DUSTB_IPVY1, p) = 0.0; P.r(DUSTB_IPVZ1, p) = 0.0;
    }
  }
  double x1 = P.r(DUSTB_IPX, p), x2 = P.r(DUSTB_IPY, p), x3 = P.r(DUSTB_IPZ, p);
  const double lx = M.s(m, X1MAX) - M.s(m, X1MIN);
  const double ly = M.s(m, X2MAX) - M.s(m, X2MIN);
  const double lz = M.s(m, X3MAX) - M.s(m, X3MIN);
  int ix = (int)((x1 - M.s(m, X1MIN) + lx) / lx) - 1;
  int iy = (int)((x2 - M.s(m, X2MIN) + ly) / ly) - 1;
  int iz = (int)((x3 - M.s(m, X3MIN) + lz) / lz) - 1;
  auto snap = [&](int off, double &x, double xa, double xb, int ipx, int irx) {
    if (off != 0) return;
    double xs = x;
    if (x < xa) xs = xa;
    else if (x >= xb) xs = nextafter(xb, xa);
    if (xs != x) { P.r(irx, p) += xs - x; P.r(ipx, p) = xs; x = xs; }
  };
  snap(ix, x1, M.s(m, X1MIN), M.s(m, X1MAX), DUSTB_IPX, DUSTB_IPX1);
  if (M.multi_d) snap(iy, x2, M.s(m, X2MIN), M.s(m, X2MAX), DUSTB_IPY, DUSTB_IPY1);
  if (M.three_d) snap(iz, x3, M.s(m, X3MIN), M.s(m, X3MAX), DUSTB_IPZ, DUSTB_IPZ1);
  if (!M.multi_d) iy = 0;
  if (!M.three_d) iz = 0;
  if (abs(ix) > 1 || abs(iy) > 1 || abs(iz) > 1) { report(err, DUSTB_ERR_ROUTE); return; }
  if (ix == 0 && iy == 0 && iz == 0) return;
  const bool lo1 = (ix < 0) && (M.s(m, X1MIN) < M.x1min + 0.5 * lx);
  const bool hi1 = (ix > 0) && (M.s(m, X1MAX) > M.x1max - 0.5 * lx);
  const bool lo2 = (iy < 0) && (M.s(m, X2MIN) < M.x2min + 0.5 * ly);
  const bool hi2 = (iy > 0) && (M.s(m, X2MAX) > M.x2max - 0.5 * ly);
  const bool lo3 = (iz < 0) && (M.s(m, X3MIN) < M.x3min + 0.5 * lz);
  const bool hi3 = (iz > 0) && (M.s(m, X3MAX) > M.x3max - 0.5 * lz);
  if (B.on && (lo1 || hi1)) {
    // a radial face (bvals_part.cpp:266-310): wrap x, shift y by the folded shear offset,
    // wrap y and z, route to the face block on the other side at the new (y, z)
    const bool cross_in = lo1;
    const double lxm = M.x1max - M.x1min;
    P.r(DUSTB_IPX, p) += cross_in ? lxm : -lxm;
    P.r(DUSTB_IPX1, p) += cross_in ? lxm : -lxm;
    const double lym = M.x2max - M.x2min;
    double ynew = P.r(DUSTB_IPY, p) + (cross_in ? -B.ysh : B.ysh);
    if (ynew < M.x2min) ynew += lym;
    if (ynew >= M.x2max) ynew -= lym;
    const double dy = ynew - P.r(DUSTB_IPY, p);
    P.r(DUSTB_IPY, p) = ynew;
    P.r(DUSTB_IPY1, p) += dy;
    const double lzm = M.x3max - M.x3min;
    if (lo3) { P.r(DUSTB_IPZ, p) += lzm; P.r(DUSTB_IPZ1, p) += lzm; }
    else if (hi3) { P.r(DUSTB_IPZ, p) -= lzm; P.r(DUSTB_IPZ1, p) -= lzm; }
    int b2 = (int)(((P.r(DUSTB_IPY, p) - M.x2min) / lym) * (double)B.nb2);
    b2 = (b2 < 0) ? 0 : ((b2 > B.nb2 - 1) ? B.nb2 - 1 : b2);
    int b3 = (int)(((P.r(DUSTB_IPZ, p) - M.x3min) / lzm) * (double)B.nb3);
    b3 = (b3 < 0) ? 0 : ((b3 > B.nb3 - 1) ? B.nb3 - 1 : b3);
    P.i(DUSTB_PGID, p) = B.sb_gid[((long long)(cross_in ? 1 : 0) * B.nb3 + b3) * B.nb2 + b2];
    return;
  }
  int gid;
  if (M.nml) {
    // (the half of the block the particle leaves from: sub-slots of finer neighbours)
    const int fx = (x1 < 0.5 * (M.s(m, X1MIN) + M.s(m, X1MAX))) ? 0 : 1;
    const int fy = (x2 < 0.5 * (M.s(m, X2MIN) + M.s(m, X2MAX))) ? 0 : 1;
    const int fz = (x3 < 0.5 * (M.s(m, X3MIN) + M.s(m, X3MAX))) ? 0 : 1;
    const int s = route_slot_ml(M, m, ix, iy, iz, fx, fy, fz);
    gid = (s < 0) ? -1 : M.nml[(long long)m * 56 + s];
  } else {
    gid = M.nghbr[(long long)m * 27 + dir_slot(ix, iy, iz)];
  }
  if (gid < 0) { report(err, DUSTB_ERR_NGHBR); return; }
  P.i(DUSTB_PGID, p) = gid;
  const double Lx = M.x1max - M.x1min, Ly = M.x2max - M.x2min, Lz = M.x3max - M.x3min;
  if (lo1) { P.r(DUSTB_IPX, p) += Lx; P.r(DUSTB_IPX1, p) += Lx; }
  else if (hi1) { P.r(DUSTB_IPX, p) -= Lx; P.r(DUSTB_IPX1, p) -= Lx; }
  if (lo2) { P.r(DUSTB_IPY, p) += Ly; P.r(DUSTB_IPY1, p) += Ly; }
  else if (hi2) { P.r(DUSTB_IPY, p) -= Ly; P.r(DUSTB_IPY1, p) -= Ly; }
  if (lo3) { P.r(DUSTB_IPZ, p) += Lz; P.r(DUSTB_IPZ1, p) += Lz; }
  else if (hi3) { P.r(DUSTB_IPZ, p) -= Lz; P.r(DUSTB_IPZ1, p) -= Lz; }
}

// ---- DepositDrag imex scatter, src/dust/dust_pm.cpp:225-274 ------------------------------
__global__ void k_scatter(PCtx P, MCtx M, Ind d, double *qdep, double a_dt, double sh,
                          unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  int m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) { report(err, DUSTB_ERR_PGID); return; }
  int ip, jp, kp; double wx[3], wy[3], wz[3];
  weights3(M, d, m, P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p) + sh * P.r(DUSTB_IPX, p),
           P.r(DUSTB_IPZ, p), ip, jp, kp, wx, wy, wz);
  if (!halo_ok(d, ip, jp, kp)) { report(err, DUSTB_ERR_HALO); return; }
  double vol = cell_vol(M, d, m);
  double cj = a_dt / (P.r(DUSTB_IPTS, p) + a_dt);
  double muc = P.r(DUSTB_IPM, p) * cj / vol;
  double vx = P.r(DUSTB_IPVX, p), vy = P.r(DUSTB_IPVY, p), vz = P.r(DUSTB_IPVZ, p);
  int clo = d.three_d ? 0 : 1, chi = d.three_d ? 2 : 1;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b] * muc;
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        atomicAdd(&qdep[d.at(m, 5, 0, kk, jj, ii)], w);
        atomicAdd(&qdep[d.at(m, 5, 1, kk, jj, ii)], w * vx);
        atomicAdd(&qdep[d.at(m, 5, 2, kk, jj, ii)], w * vy);
        atomicAdd(&qdep[d.at(m, 5, 3, kk, jj, ii)], w * vz);
      }
    }
}

// ---- ghost exchanges (pull form, one thread per destination cell) -----------------------
// RecvAndSumDeposit (src/bvals/bvals_dep.cpp:457-560): receiver active strips on side o
// (InitRecvIndices :281-297) += the neighbour's ghost cells at index - o*nx, in
// NeighborIndex order.

// The active cells within ng of a face of their block (the only ones a neighbour's ghost
// cells reach), enumerated per block: the near x3 planes whole (zn of them), then in each of
// the zin inner planes its near x2 rows whole (yn) and, in each of its yin inner rows, the xn
// cells near the x1 faces.  A dimension the mesh lacks has no near part (zn = 0, zin = nx3).
struct Shell { int zn, zin, yn, yin, xn, xin, zoff, yoff; long long per; };

__host__ __device__ inline Shell make_shell(const Ind &d) {
  Shell h;
  const int g2 = 2 * d.ng;
  h.xn = d.nx1 < g2 ? d.nx1 : g2;
  h.xin = d.nx1 - h.xn;
  h.yn = d.multi_d ? (d.nx2 < g2 ? d.nx2 : g2) : 0;
  h.yin = d.nx2 - h.yn;
  h.zn = d.three_d ? (d.nx3 < g2 ? d.nx3 : g2) : 0;
  h.zin = d.nx3 - h.zn;
  h.yoff = d.multi_d ? d.ng : 0;
  h.zoff = d.three_d ? d.ng : 0;
  h.per = (long long)h.zn * d.nx2 * d.nx1 +
          (long long)h.zin * ((long long)h.yn * d.nx1 + (long long)h.yin * h.xn);
  return h;
}

// t in [0, per) -> the cell's offsets from (ks, js, is)
__device__ __forceinline__ void shell_cell(const Ind &d, const Shell &h, long long t, int &k,
                                           int &j, int &i) {
  const long long plane = (long long)d.nx2 * d.nx1;
  if (t < (long long)h.zn * plane) {
    const int z = (int)(t / plane);
    const long long r = t - z * plane;
    k = z < d.ng ? z : z + h.zin;
    j = (int)(r / d.nx1);
    i = (int)(r - (long long)j * d.nx1);
    return;
  }
  t -= (long long)h.zn * plane;
  const long long inner = (long long)h.yn * d.nx1 + (long long)h.yin * h.xn;
  const int z = (int)(t / inner);
  long long r = t - z * inner;
  k = h.zoff + z;
  if (r < (long long)h.yn * d.nx1) {
    const int y = (int)(r / d.nx1);
    j = y < d.ng ? y : y + h.yin;
    i = (int)(r - (long long)y * d.nx1);
    return;
  }
  r -= (long long)h.yn * d.nx1;
  const int y = (int)(r / h.xn);
  const int u = (int)(r - (long long)y * h.xn);
  j = h.yoff + y;
  i = u < d.ng ? u : u + h.xin;
}

// fold: fold the ghost deposits beyond physical x3 faces back into the mirrored active cells
__global__ void k_ghost_add(Ind d, const int *nghbr, int gids, double *a, int nvar, int fold,
                            SBox B) {
  int m, k, j, i;
  const Shell sh = make_shell(d);
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long ncell = (long long)d.nmb * sh.per;
  int v = (int)(idx / ncell);
  if (v >= nvar) return;
  {
    const long long r = idx - (long long)v * ncell;
    m = (int)(r / sh.per);
    shell_cell(d, sh, r - (long long)m * sh.per, k, j, i);
    k += d.ks; j += d.js; i += d.is;
  }
  const int ng1 = d.ng - 1;
  const int ndir = d.three_d ? 26 : (d.multi_d ? 8 : 2);
  const long long at = d.at(m, nvar, v, k, j, i);
  double val = a[at];
  for (int n = 0; n < ndir; ++n) {
    const int o1 = kDirOrder[n][0], o2 = kDirOrder[n][1], o3 = kDirOrder[n][2];
    if (o1 > 0 && i < d.ie - ng1) continue;
    if (o1 < 0 && i > d.is + ng1) continue;
    if (o2 > 0 && j < d.je - ng1) continue;
    if (o2 < 0 && j > d.js + ng1) continue;
    if (o3 > 0 && k < d.ke - ng1) continue;
    if (o3 < 0 && k > d.ks + ng1) continue;
    const int src = nghbr[(long long)m * 27 + dir_slot(o1, o2, o3)] - gids;
    if (src < 0 || src >= d.nmb || B.crossing(m, o1)) continue;
    val += a[d.at(src, nvar, v, k - o3 * d.nx3, j - o2 * d.nx2, i - o1 * d.nx1)];
  }
  if (fold && d.three_d) {
    // a physical x3 face (no neighbour across it): the ghost plane ks-1-t (ke+1+t) folds into
    // the active plane ks+t (ke-t); the block's own column, then its x1/x2 neighbours'
    // ghost strips that face this cell, in NeighborIndex order
    for (int side = 0; side < 2; ++side) {
      const int o3 = side ? 1 : -1;
      if (side == 0 ? (k > d.ks + ng1) : (k < d.ke - ng1)) continue;
      if (nghbr[(long long)m * 27 + dir_slot(0, 0, o3)] >= 0) continue;
      const int kg = side ? 2 * d.ke + 1 - k : 2 * d.ks - 1 - k;
      val += a[d.at(m, nvar, v, kg, j, i)];
      for (int n = 0; n < ndir; ++n) {
        const int o1 = kDirOrder[n][0], o2 = kDirOrder[n][1];
        if (kDirOrder[n][2] != 0) continue;
        if (o1 > 0 && i < d.ie - ng1) continue;
        if (o1 < 0 && i > d.is + ng1) continue;
        if (o2 > 0 && j < d.je - ng1) continue;
        if (o2 < 0 && j > d.js + ng1) continue;
        const int src = nghbr[(long long)m * 27 + dir_slot(o1, o2, 0)] - gids;
        if (src < 0 || src >= d.nmb || B.crossing(m, o1)) continue;
        val += a[d.at(src, nvar, v, kg, j - o2 * d.nx2, i - o1 * d.nx1)];
      }
    }
  }
  a[at] = val;
}

// shear-periodic x1 faces: the remapped ghost cells beyond them, their sum added as
// DepRemapPlan's GeneralApply adds it, after the exchange above (a pass of its own over the
// strips of active cells next to the faces: the exchange reads only ghost cells, this one
// too, so the order of the additions is that of one pass)
__global__ void k_shear_add(Ind d, SBox B, double *a, int nvar) {
  const int ng = d.ng, ng1 = d.ng - 1;
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int c = (int)(idx % (2 * ng)); idx /= 2 * ng;
  const int j = (int)(idx % d.nx2) + d.js; idx /= d.nx2;
  const int k = (int)(idx % d.nx3) + d.ks; idx /= d.nx3;
  const int v = (int)(idx % nvar); idx /= nvar;
  if (idx >= d.nmb) return;
  const int m = (int)idx;
  const int faces = B.faces(m);
  if (!faces) return;
  // strip column c: the inner strip's is + c, else the outer strip's (once if they overlap)
  const int i = (c < ng) ? d.is + c : d.ie - ng1 + (c - ng);
  if (c >= ng && i <= d.is + ng1) return;
  const bool inner = (faces & 1) && i <= d.is + ng1, outer = (faces & 2) && i >= d.ie - ng1;
  if (!inner && !outer) return;
  const long long at = d.at(m, nvar, v, k, j, i);
  a[at] += shear_add_sum(B, d, a, nvar, m, v, k, j, i);
}

// the general deposit remap of a refined mesh (GeneralApply, bvals_dep_general.cpp:1135-1175):
// one thread per (target cell, variable), its sources summed in list order and added once.
// Sources are ghost cells and targets active cells, so no thread reads what another writes.
__global__ void k_dep_plan_apply(int nseg, const int *__restrict__ tgt, const int *__restrict__ ptr,
                                 const int *__restrict__ src, const double *__restrict__ w,
                                 double *a, int nvar, long long ncell) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nseg * nvar) return;
  const int s = (int)(t / nvar), v = (int)(t - (long long)s * nvar);
  double sum = 0.0;
  for (int e = ptr[s]; e < ptr[s + 1]; ++e) {
    const long long q = src[e];
    const long long sm = q / ncell;
    sum += w[e] * a[(sm * nvar + v) * ncell + (q - sm * ncell)];
  }
  const long long c = tgt[s];
  const long long tm = c / ncell;
  a[(tm * nvar + v) * ncell + (c - tm * ncell)] += sum;
}

// copy exchange: every ghost cell <- the neighbour's active cell at index - o*nx
__global__ void k_ghost_copy(Ind d, const int *nghbr, int gids, double *a, int nvar) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long per = d.cells();
  long long tot = per * d.nmb;
  if (idx >= tot) return;
  int m = (int)(idx / per);
  long long r = idx - (long long)m * per;
  int i = (int)(r % d.n1); r /= d.n1;
  int j = (int)(r % d.n2);
  int k = (int)(r / d.n2);
  int o1 = (i < d.is) ? -1 : ((i > d.ie) ? 1 : 0);
  int o2 = (j < d.js) ? -1 : ((j > d.je) ? 1 : 0);
  int o3 = (k < d.ks) ? -1 : ((k > d.ke) ? 1 : 0);
  if (o1 == 0 && o2 == 0 && o3 == 0) return;
  const int src = nghbr[(long long)m * 27 + dir_slot(o1, o2, o3)] - gids;
  if (src < 0 || src >= d.nmb) return;
  for (int v = 0; v < nvar; ++v)
    a[d.at(m, nvar, v, k, j, i)] = a[d.at(src, nvar, v, k - o3 * d.nx3, j - o2 * d.nx2, i - o1 * d.nx1)];
}

// UstarX3BCs, src/dust/dust_tasks.cpp:445-469
__global__ void k_x3_bcs(Ind d, const int *nghbr, double *a, int refl) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long per = (long long)d.ng * d.n2 * d.n1;
  if (idx >= per * d.nmb) return;
  int m = (int)(idx / per);
  long long r = idx - (long long)m * per;
  int i = (int)(r % d.n1); r /= d.n1;
  int j = (int)(r % d.n2);
  int g = (int)(r / d.n2);
  const bool lo_face = nghbr[(long long)m * 27 + dir_slot(0, 0, -1)] < 0;
  const bool hi_face = nghbr[(long long)m * 27 + dir_slot(0, 0, 1)] < 0;
  if (lo_face) {
    int kg = d.ks - 1 - g, kc = refl ? (d.ks + g) : d.ks;
    for (int v = 0; v < 3; ++v)
      a[d.at(m, 3, v, kg, j, i)] = (refl && v == 2) ? -a[d.at(m, 3, v, kc, j, i)] : a[d.at(m, 3, v, kc, j, i)];
  }
  if (hi_face) {
    int kg = d.ke + 1 + g, kc = refl ? (d.ke - g) : d.ke;
    for (int v = 0; v < 3; ++v)
      a[d.at(m, 3, v, kg, j, i)] = (refl && v == 2) ? -a[d.at(m, 3, v, kc, j, i)] : a[d.at(m, 3, v, kc, j, i)];
  }
}

// ---- solve (dust_pm.cpp:426-436) --------------------------------------------------------
__global__ void k_solve_ustar(Ind d, const double *u0, int nv, const double *qdep, double *us,
                              int br) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  double q0 = br ? qdep[d.at(m, 5, 0, k, j, i)] : 0.0;
  double denom = 1.0 / (u0[d.at(m, nv, 0, k, j, i)] + q0);
  for (int v = 0; v < 3; ++v) {
    double qv = br ? qdep[d.at(m, 5, 1 + v, k, j, i)] : 0.0;
    us[d.at(m, 3, v, k, j, i)] = (u0[d.at(m, nv, 1 + v, k, j, i)] + qv) * denom;
  }
}

// ---- PointOperatorParticles, src/dust/dust_solver.cpp:151-201 ---------------------------
__global__ void k_operator(PCtx P, MCtx M, Ind d, const double *field, double *result,
                           double a_dt, double sh, unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  int m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) { report(err, DUSTB_ERR_PGID); return; }
  int ip, jp, kp; double wx[3], wy[3], wz[3];
  weights3(M, d, m, P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p) + sh * P.r(DUSTB_IPX, p),
           P.r(DUSTB_IPZ, p), ip, jp, kp, wx, wy, wz);
  if (!halo_ok(d, ip, jp, kp)) { report(err, DUSTB_ERR_HALO); return; }
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  int clo = d.three_d ? 0 : 1, chi = d.three_d ? 2 : 1;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b];
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        g0 += w * field[d.at(m, 3, 0, kk, jj, ii)];
        g1 += w * field[d.at(m, 3, 1, kk, jj, ii)];
        g2 += w * field[d.at(m, 3, 2, kk, jj, ii)];
      }
    }
  double vol = cell_vol(M, d, m);
  double cj = a_dt / (P.r(DUSTB_IPTS, p) + a_dt);
  double fac = P.r(DUSTB_IPM, p) * cj / vol;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b] * fac;
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        atomicAdd(&result[d.at(m, 3, 0, kk, jj, ii)], w * g0);
        atomicAdd(&result[d.at(m, 3, 1, kk, jj, ii)], w * g1);
        atomicAdd(&result[d.at(m, 3, 2, kk, jj, ii)], w * g2);
      }
    }
}

// dust_applya_dc, src/dust/dust_solver.cpp:243-252
__global__ void k_dc_correct(Ind d, const double *u0, int nv, const double *qdep,
                             const double *result, double *field) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  double rho = u0[d.at(m, nv, 0, k, j, i)];
  double pinv = 1.0 / (rho + qdep[d.at(m, 5, 0, k, j, i)]);
  for (int v = 0; v < 3; ++v) {
    long long a = d.at(m, 3, v, k, j, i);
    double av = result[a] + rho * field[a];
    double rv = u0[d.at(m, nv, 1 + v, k, j, i)] + qdep[d.at(m, 5, 1 + v, k, j, i)] - av;
    field[a] += pinv * rv;
  }
}

// ---- GatherKickPMBR, src/dust/dust_pm.cpp:500-564 ----------------------------------------
__global__ void k_gather_kick(PCtx P, MCtx M, Ind d, const double *us, double *dmom, double a_dt,
                              double sh, int br, unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  int m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) { report(err, DUSTB_ERR_PGID); return; }
  int ip, jp, kp; double wx[3], wy[3], wz[3];
  weights3(M, d, m, P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p) + sh * P.r(DUSTB_IPX, p),
           P.r(DUSTB_IPZ, p), ip, jp, kp, wx, wy, wz);
  if (!halo_ok(d, ip, jp, kp)) { report(err, DUSTB_ERR_HALO); return; }
  double ux = 0.0, uy = 0.0, uz = 0.0;
  int clo = d.three_d ? 0 : 1, chi = d.three_d ? 2 : 1;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b];
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        ux += w * us[d.at(m, 3, 0, kk, jj, ii)];
        uy += w * us[d.at(m, 3, 1, kk, jj, ii)];
        uz += w * us[d.at(m, 3, 2, kk, jj, ii)];
      }
    }
  double cj = a_dt / (P.r(DUSTB_IPTS, p) + a_dt);
  double dvx = cj * (ux - P.r(DUSTB_IPVX, p));
  double dvy = cj * (uy - P.r(DUSTB_IPVY, p));
  double dvz = cj * (uz - P.r(DUSTB_IPVZ, p));
  P.r(DUSTB_IPVX, p) += dvx; P.r(DUSTB_IPVY, p) += dvy; P.r(DUSTB_IPVZ, p) += dvz;
  P.r(DUSTB_IPRX, p) = dvx / a_dt; P.r(DUSTB_IPRY, p) = dvy / a_dt; P.r(DUSTB_IPRZ, p) = dvz / a_dt;
  if (!br) return;
  double vol = cell_vol(M, d, m);
  double fac = -P.r(DUSTB_IPM, p) / vol;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b] * fac;
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        atomicAdd(&dmom[d.at(m, 3, 0, kk, jj, ii)], w * dvx);
        atomicAdd(&dmom[d.at(m, 3, 1, kk, jj, ii)], w * dvy);
        atomicAdd(&dmom[d.at(m, 3, 2, kk, jj, ii)], w * dvz);
      }
    }
}

// ---- ApplyPMBR, src/dust/dust_pm.cpp:649-708 ---------------------------------------------
__device__ __forceinline__ bool center_cell(const PCtx &P, const MCtx &M, const Ind &d, int p,
                                            int &m, int &ip, int &jp, int &kp) {
  m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) return false;
  double w[3];
  pm_weights(P.r(DUSTB_IPX, p), M.s(m, X1MIN), M.s(m, X1MAX), d.nx1, d.is, M.scheme, ip, w);
  pm_weights(P.r(DUSTB_IPY, p), M.s(m, X2MIN), M.s(m, X2MAX), d.nx2, d.js, M.scheme, jp, w);
  if (d.three_d) pm_weights(P.r(DUSTB_IPZ, p), M.s(m, X3MIN), M.s(m, X3MAX), d.nx3, d.ks, M.scheme, kp, w);
  else kp = d.ks;
  return halo_ok(d, ip, jp, kp);
}

__global__ void k_center_mass(PCtx P, MCtx M, Ind d, double *res, double a_dt, unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  if (P.r(DUSTB_IPM, p) <= 0.0) return;
  int m, ip, jp, kp;
  if (!center_cell(P, M, d, p, m, ip, jp, kp)) { report(err, DUSTB_ERR_HALO); return; }
  double vol = cell_vol(M, d, m);
  atomicAdd(&res[d.at(m, 4, 3, kp, jp, ip)],
            P.r(DUSTB_IPM, p) * (a_dt / (P.r(DUSTB_IPTS, p) + a_dt)) / vol);
}

__global__ void k_consistent_gas(Ind d, double *u0, int nv, const double *us, const double *qdep,
                                 double *dmom, double *res, double inv_adt) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  const double rho = u0[d.at(m, nv, 0, k, j, i)], qt = res[d.at(m, 4, 3, k, j, i)];
  const double q = qdep[d.at(m, 5, 0, k, j, i)];
  for (int v = 0; v < 3; ++v) {
    long long a3 = d.at(m, 3, v, k, j, i);
    long long au = d.at(m, nv, 1 + v, k, j, i);
    double dgas = dmom[a3];
    if (qt > 0.0) {
      const double g = rho * us[a3] - u0[au];
      const double r = (dmom[a3] - g) / (rho + q);
      dgas = g + rho * r;
      res[d.at(m, 4, v, k, j, i)] = r * q / qt;
    }
    u0[au] += dgas;
    dmom[a3] = dgas * inv_adt;
  }
}

__global__ void k_consistent_dust(PCtx P, MCtx M, Ind d, const double *res, double a_dt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  if (P.r(DUSTB_IPM, p) <= 0.0) return;
  int m, ip, jp, kp;
  if (!center_cell(P, M, d, p, m, ip, jp, kp)) return;
  const double cj = a_dt / (P.r(DUSTB_IPTS, p) + a_dt);
  for (int v = 0; v < 3; ++v) {
    const double dv = cj * res[d.at(m, 4, v, kp, jp, ip)];
    P.r(DUSTB_IPVX + 2 * v, p) += dv;
    P.r(DUSTB_IPRX + v, p) += dv / a_dt;
  }
}

__global__ void k_pmbr(Ind d, double *u0, int nv, double *dmom, double inv_adt) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  for (int v = 0; v < 3; ++v) {
    long long a3 = d.at(m, 3, v, k, j, i);
    u0[d.at(m, nv, 1 + v, k, j, i)] += dmom[a3];
    dmom[a3] *= inv_adt;
  }
}

// ---- reductions: newdt, stopping times ---------------------------------------------------
__device__ __forceinline__ void atomic_min_pos(double *a, double v) {
  atomicMin((unsigned long long *)a, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_pos(double *a, double v) {
  atomicMax((unsigned long long *)a, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_set(double *a, double v0, int two, double v1) {
  a[0] = v0;
  if (two) a[1] = v1;
}

__global__ void k_newdt(PCtx P, MCtx M, Ind d, int shear3d, double qo, double *out) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  double t = (double)FLT_MAX;
  if (p < P.npart) {
    int m = P.i(DUSTB_PGID, p) - M.gids;
    if (block_ok(d, m)) {
      double vy = P.r(DUSTB_IPVY, p);
      if (shear3d) vy -= qo * P.r(DUSTB_IPX, p);
      t = fmin(M.s(m, DX1) / fmax(fabs(P.r(DUSTB_IPVX, p)), 1.0e-30), t);
      t = fmin(M.s(m, DX2) / fmax(fabs(vy), 1.0e-30), t);
      if (d.three_d) t = fmin(M.s(m, DX3) / fmax(fabs(P.r(DUSTB_IPVZ, p)), 1.0e-30), t);
    }
  }
  for (int o = 16; o > 0; o >>= 1) t = fmin(t, __shfl_xor_sync(0xffffffffu, t, o));
  if ((threadIdx.x & 31) == 0) atomic_min_pos(out, t);
}

__global__ void k_scale(double *a, double s) { a[0] = s * a[0]; }

__global__ void k_tstop(PCtx P, double *out, unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  double mx = 0.0, mn = DBL_MAX;
  if (p < P.npart) {
    double ts = P.r(DUSTB_IPTS, p);
    int s = P.i(DUSTB_PSP, p);
    bool bad = (s < 0 || !isfinite(ts) || !(ts > 0.0));
    if (bad) report(err, DUSTB_ERR_TSTOP);
    mx = bad ? DBL_MAX : ts;
    mn = (ts > 0.0) ? ts : DBL_MAX;
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) { atomic_max_pos(&out[0], mx); atomic_min_pos(&out[1], mn); }
}

// ---- pc2 ---------------------------------------------------------------------------------
// DepositDrag pc2 predictor, src/dust/dust_pm.cpp:141-193
__global__ void k_pc2_predictor(PCtx P, MCtx M, Ind d, const double *uold, int nv, double *qdep,
                                double dt, int rate_dep, unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  int m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) { report(err, DUSTB_ERR_PGID); return; }
  int ip, jp, kp; double wx[3], wy[3], wz[3];
  weights3(M, d, m, P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p), P.r(DUSTB_IPZ, p), ip, jp, kp, wx, wy, wz);
  if (!halo_ok(d, ip, jp, kp)) { report(err, DUSTB_ERR_HALO); return; }
  double ugx = 0.0, ugy = 0.0, ugz = 0.0;
  int clo = d.three_d ? 0 : 1, chi = d.three_d ? 2 : 1;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b];
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        double invrho = 1.0 / uold[d.at(m, nv, 0, kk, jj, ii)];
        ugx += w * uold[d.at(m, nv, 1, kk, jj, ii)] * invrho;
        ugy += w * uold[d.at(m, nv, 2, kk, jj, ii)] * invrho;
        ugz += w * uold[d.at(m, nv, 3, kk, jj, ii)] * invrho;
      }
    }
  double vol = cell_vol(M, d, m);
  double rate = P.r(DUSTB_IPM, p) / (P.r(DUSTB_IPTS, p) * vol);
  double gx = -dt * rate * (ugx - P.r(DUSTB_IPVX, p));
  double gy = -dt * rate * (ugy - P.r(DUSTB_IPVY, p));
  double gz = -dt * rate * (ugz - P.r(DUSTB_IPVZ, p));
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b];
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        atomicAdd(&qdep[d.at(m, 5, 1, kk, jj, ii)], w * gx);
        atomicAdd(&qdep[d.at(m, 5, 2, kk, jj, ii)], w * gy);
        atomicAdd(&qdep[d.at(m, 5, 3, kk, jj, ii)], w * gz);
        if (rate_dep) atomicAdd(&qdep[d.at(m, 5, 4, kk, jj, ii)], w * rate);
      }
    }
}

// UpdateStiffness's maximum of qdep4/rho (dust_pm.cpp:295-301), before the damping
__global__ void k_pc2_rate_max(Ind d, const double *u0, int nv, const double *qdep, double *out) {
  int m, k, j, i;
  double r = 0.0;
  if (active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i))
    r = qdep[d.at(m, 5, 4, k, j, i)] / u0[d.at(m, nv, 0, k, j, i)];
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  if ((threadIdx.x & 31) == 0 && r > 0.0) atomic_max_pos(out, r);
}

// dust_pc2_apply_predictor, dust_pm.cpp:387-402
__global__ void k_pc2_apply(Ind d, double *u0, int nv, double *qdep, double dt, int damp) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  if (damp) {
    const double chi = dt * qdep[d.at(m, 5, 4, k, j, i)] / u0[d.at(m, nv, 0, k, j, i)];
    if (chi > 1.0) {
      const double s = 1.0 / chi;
      for (int v = 1; v <= 3; ++v) qdep[d.at(m, 5, v, k, j, i)] *= s;
    }
  }
  for (int v = 1; v <= 3; ++v) u0[d.at(m, nv, v, k, j, i)] += qdep[d.at(m, 5, v, k, j, i)];
}

// dust_gas_midpoint, dust_push.cpp:53-59 (ghosts included)
__global__ void k_pc2_midpoint(Ind d, const double *u0, const double *u1, int nv, double *us) {
  long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long per = d.cells();
  if (idx >= per * d.nmb) return;
  int m = (int)(idx / per);
  long long c = idx - (long long)m * per;
  const long long b0 = ((long long)m * nv) * per + c;
  double inv = 1.0 / (u1[b0] + u0[b0]);
  for (int v = 0; v < 3; ++v) {
    long long bv = ((long long)m * nv + 1 + v) * per + c;
    us[((long long)m * 3 + v) * per + c] = (u1[bv] + u0[bv]) * inv;
  }
}

// dust_pc2_advance, src/dust/dust_push.cpp:132-245
__global__ void k_pc2_advance(PCtx P, MCtx M, Ind d, const double *us, double *dmom, double dt,
                              int br, int sbox, int strat, double q, double om, double aphi,
                              unsigned *err) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  int m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) { report(err, DUSTB_ERR_PGID); return; }
  const bool three_d = d.three_d;
  double x0 = P.r(DUSTB_IPX1, p), y0 = P.r(DUSTB_IPY1, p), z0 = P.r(DUSTB_IPZ1, p);
  double vx0 = P.r(DUSTB_IPVX1, p), vy0 = P.r(DUSTB_IPVY1, p), vz0 = P.r(DUSTB_IPVZ1, p);
  double xh = x0 + 0.5 * dt * vx0;
  double yh = y0 + 0.5 * dt * (vy0 - ((sbox && three_d) ? q * om * x0 : 0.0));
  double zh = three_d ? z0 + 0.5 * dt * vz0 : z0;
  double yg = yh + ((sbox && three_d) ? q * om * xh * 0.5 * dt : 0.0);
  int ip, jp, kp; double wx[3], wy[3], wz[3];
  weights3(M, d, m, xh, yg, zh, ip, jp, kp, wx, wy, wz);
  if (!halo_ok(d, ip, jp, kp)) { report(err, DUSTB_ERR_HALO); return; }
  double ugx = 0.0, ugy = 0.0, ugz = 0.0;
  int clo = three_d ? 0 : 1, chi = three_d ? 2 : 1;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b];
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        ugx += w * us[d.at(m, 3, 0, kk, jj, ii)];
        ugy += w * us[d.at(m, 3, 1, kk, jj, ii)];
        ugz += w * us[d.at(m, 3, 2, kk, jj, ii)];
      }
    }
  double h = 0.5 * dt;
  double lambda = h / P.r(DUSTB_IPTS, p);
  double aa = 1.0 + lambda;
  double rx = vx0 + lambda * ugx, ry = vy0 + lambda * ugy, rz = vz0 + lambda * ugz;
  double vxh, vyh, vzh;
  if (sbox && three_d) {
    double cxy = 2.0 * h * om, cyx = h * (2.0 - q) * om;
    double det = aa * aa + cxy * cyx;
    vxh = (aa * rx + cxy * ry) / det;
    vyh = (aa * ry - cyx * rx) / det;
    if (strat) rz -= h * (om * om) * zh;
    vzh = rz / aa;
  } else if (sbox) {
    double cxz = 2.0 * h * om, czx = h * (2.0 - q) * om;
    double det = aa * aa + cxz * czx;
    if (aphi != 0.0) rz += h * aphi;
    vxh = (aa * rx + cxz * rz) / det;
    vzh = (aa * rz - czx * rx) / det;
    vyh = ry / aa;
  } else {
    vxh = rx / aa; vyh = ry / aa; vzh = rz / aa;
  }
  P.r(DUSTB_IPVX, p) = 2.0 * vxh - vx0;
  P.r(DUSTB_IPVY, p) = 2.0 * vyh - vy0;
  P.r(DUSTB_IPVZ, p) = 2.0 * vzh - vz0;
  P.r(DUSTB_IPX, p) = x0 + dt * vxh;
  P.r(DUSTB_IPY, p) = y0 + dt * (vyh - ((sbox && three_d) ? q * om * xh : 0.0));
  if (three_d) P.r(DUSTB_IPZ, p) = z0 + dt * vzh;
  P.r(DUSTB_IPX1, p) = xh; P.r(DUSTB_IPY1, p) = yh; P.r(DUSTB_IPZ1, p) = zh;
  double dvx = dt * (ugx - vxh) / P.r(DUSTB_IPTS, p);
  double dvy = dt * (ugy - vyh) / P.r(DUSTB_IPTS, p);
  double dvz = dt * (ugz - vzh) / P.r(DUSTB_IPTS, p);
  P.r(DUSTB_IPRX, p) = dvx; P.r(DUSTB_IPRY, p) = dvy; P.r(DUSTB_IPRZ, p) = dvz;
  if (!br) return;
  double vol = cell_vol(M, d, m);
  double fac = -P.r(DUSTB_IPM, p) / vol;
  for (int c = clo; c <= chi; ++c)
    for (int b = 0; b < 3; ++b) {
      double wcb = wz[c] * wy[b] * fac;
      if (wcb == 0.0) continue;
      for (int a = 0; a < 3; ++a) {
        double w = wcb * wx[a];
        int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        atomicAdd(&dmom[d.at(m, 3, 0, kk, jj, ii)], w * dvx);
        atomicAdd(&dmom[d.at(m, 3, 1, kk, jj, ii)], w * dvy);
        atomicAdd(&dmom[d.at(m, 3, 2, kk, jj, ii)], w * dvz);
      }
    }
}

// dust_pc2_commit, dust_pm.cpp:596-601
__global__ void k_pc2_commit(Ind d, double *u0, int nv, const double *dmom, const double *qdep,
                             double wpred) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  for (int v = 0; v < 3; ++v)
    u0[d.at(m, nv, 1 + v, k, j, i)] += dmom[d.at(m, 3, v, k, j, i)] - wpred * qdep[d.at(m, 5, 1 + v, k, j, i)];
}

// ---- ParticleHistory (the phst row), src/dust/dust_science.cpp:391-482 ------------------
constexpr int kPhstChunk = 4096, kPhstSums = 7;

// the particle sums of one chunk of 4096 particles, in particle order (dust_science.cpp:400-413)
__global__ void k_phst_chunks(PCtx P, int zc, double *part, int nchunk) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunk) return;
  double a[kPhstSums] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const int p0 = c * kPhstChunk, p1 = min(p0 + kPhstChunk, P.npart);
  for (int p = p0; p < p1; ++p) {
    const double m = P.r(DUSTB_IPM, p);
    if (m == 0.0) continue;                        // outflow tombstones
    const double v1 = P.r(DUSTB_IPVX, p), v2 = P.r(DUSTB_IPVY, p), v3 = P.r(DUSTB_IPVZ, p);
    const double z = P.r(zc, p);
    a[0] += 1.0;
    a[1] += m;
    a[2] += m * v1; a[3] += m * v2; a[4] += m * v3;
    a[5] += 0.5 * m * (v1 * v1 + v2 * v2 + v3 * v3);
    a[6] += m * z * z;
  }
  for (int q = 0; q < kPhstSums; ++q) part[(long long)c * kPhstSums + q] = a[q];
}

// the chunks summed in order (the host loop of dust_science.cpp:415-416), one thread
__global__ void k_phst_sums(const double *part, int nchunk, const double *chi, int br,
                            double *row) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double s[kPhstSums] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int c = 0; c < nchunk; ++c)
    for (int q = 0; q < kPhstSums; ++q) s[q] += part[(long long)c * kPhstSums + q];
  for (int q = 0; q < 6; ++q) row[q] = s[q];
  row[6] = (s[1] > 0.0) ? sqrt(s[6] / s[1]) : 0.0;
  row[12] = (br && chi) ? *chi : -1.0;
  row[13] = -1.0;
  row[14] = 0.0;
  row[15] = 0.0;
}

// the mass component of DepositPointScienceFields (src/dust/dust_gravity_points.cpp:277-304):
// m/V with the deposit weights into the block's cells, ghost cells included
__global__ void k_mass_deposit(PCtx P, MCtx M, Ind d, double *f, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const double mass = P.r(DUSTB_IPM, p);
  if (mass == 0.0) return;
  const int m = P.i(DUSTB_PGID, p) - M.gids;
  if (!block_ok(d, m)) { report(err, DUSTB_ERR_PGID); return; }
  int ip, jp, kp; double wx[3], wy[3], wz[3];
  weights3(M, d, m, P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p), P.r(DUSTB_IPZ, p), ip, jp, kp, wx, wy, wz);
  if (!halo_ok(d, ip, jp, kp)) { report(err, DUSTB_ERR_HALO); return; }
  const double density = mass / cell_vol(M, d, m);
  for (int c = 0; c < 3; ++c)
    for (int b = 0; b < 3; ++b)
      for (int a = 0; a < 3; ++a) {
        const double w = density * wz[c] * wy[b] * wx[a];
        if (w == 0.0) continue;
        atomicAdd(&f[d.at(m, 1, 0, kp + c - 1, jp + b - 1, ip + a - 1)], w);
      }
}

// the densest active cell (dust_science.cpp:428-441): per block of threads the largest value
// and, among equal values, the smallest cell index q = ((m nx3 + k) nx2 + j) nx1 + i
__device__ __forceinline__ void better(double &bv, long long &bq, double v, long long q) {
  if (v > bv || (v == bv && q < bq && bq >= 0)) { bv = v; bq = q; }
}
__global__ void k_argmax_blocks(Ind d, const double *f, double *bval, long long *bloc) {
  __shared__ double sv[256];
  __shared__ long long sq[256];
  const long long ncell = (long long)d.nx1 * d.nx2 * d.nx3;
  double v = 0.0;
  long long q = -1;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < ncell * d.nmb;
       x += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(x / ncell);
    const long long r = x - (long long)m * ncell;
    const int k = (int)(r / ((long long)d.nx1 * d.nx2)), j = (int)((r / d.nx1) % d.nx2), i = (int)(r % d.nx1);
    better(v, q, f[d.at(m, 1, 0, d.ks + k, d.js + j, d.is + i)], x);
  }
  sv[threadIdx.x] = v; sq[threadIdx.x] = q;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      double bv = sv[threadIdx.x]; long long bq = sq[threadIdx.x];
      const double ov = sv[threadIdx.x + o]; const long long oq = sq[threadIdx.x + o];
      if (oq >= 0) better(bv, bq, ov, oq);
      sv[threadIdx.x] = bv; sq[threadIdx.x] = bq;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) { bval[blockIdx.x] = sv[0]; bloc[blockIdx.x] = sq[0]; }
}
__global__ void k_argmax_final(Ind d, MCtx M, const double *bval, const long long *bloc,
                               int nb, double *row) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double v = 0.0;
  long long q = -1;
  for (int b = 0; b < nb; ++b) if (bloc[b] >= 0) better(v, q, bval[b], bloc[b]);
  row[7] = (q >= 0 && v > 0.0) ? v : 0.0;
  row[8] = row[9] = row[10] = 0.0;
  row[11] = -1.0;
  if (q >= 0 && v > 0.0) {
    const long long ncell = (long long)d.nx1 * d.nx2 * d.nx3;
    const int m = (int)(q / ncell);
    const long long r = q - (long long)m * ncell;
    const int k = (int)(r / ((long long)d.nx1 * d.nx2)), j = (int)((r / d.nx1) % d.nx2), i = (int)(r % d.nx1);
    row[8] = M.s(m, X1MIN) + (i + 0.5) * M.s(m, DX1);
    row[9] = M.s(m, X2MIN) + (j + 0.5) * M.s(m, DX2);
    row[10] = d.three_d ? M.s(m, X3MIN) + (k + 0.5) * M.s(m, DX3) : 0.0;
    row[11] = 0.0;                                 // single level: the root
  }
}

// ---- point-particle fields for self-gravity and outputs, src/dust/dust_gravity_points.cpp --
// A 3-D point particle the transfers accept (:216-223, :282-287): a finite mass (gravity: also
// >= 0), an owner block in the pack, a finite position and a stencil inside the padded block.
// Massless particles (outflow tombstones) contribute nothing; the science fields also skip
// the particles of other species.  A rejected particle sets DUSTB_ERR_POINT (the reference
// aborts the run).
__device__ __forceinline__ bool point_stencil(const PCtx &P, const MCtx &M, const Ind &d, int p,
                                              int &m, int &ip, int &jp, int &kp, double wx[3],
                                              double wy[3], double wz[3]) {
  m = P.i(DUSTB_PGID, p) - M.gids;
  const double x = P.r(DUSTB_IPX, p), y = P.r(DUSTB_IPY, p), z = P.r(DUSTB_IPZ, p);
  if (!block_ok(d, m) || !isfinite(x) || !isfinite(y) || !isfinite(z)) return false;
  weights3(M, d, m, x, y, z, ip, jp, kp, wx, wy, wz);
  return ip >= 1 && ip < d.n1 - 1 && jp >= 1 && jp < d.n2 - 1 && kp >= 1 && kp < d.n3 - 1;
}

// DepositPointGravityDensity (:215-245; gravity = 1: density only, mass >= 0) and
// DepositPointScienceFields (:257-304; ncomp 1 or 4: m/V and m v/V, one species or all):
// the density with the deposit weights into the owner block's cells, ghost cells included
__global__ void k_point_deposit(PCtx P, MCtx M, Ind d, double *f, int ncomp, int species,
                                int gravity, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const double mass = P.r(DUSTB_IPM, p);
  if (gravity) {
    if (!(mass >= 0.0) || !isfinite(mass)) { report(err, DUSTB_ERR_POINT); return; }
    if (mass == 0.0) return;
  } else {
    if (mass == 0.0) return;
    if (species >= 0 && P.i(DUSTB_PSP, p) != species) return;
    if (!isfinite(mass)) { report(err, DUSTB_ERR_POINT); return; }
  }
  int m, ip, jp, kp; double wx[3], wy[3], wz[3];
  if (!point_stencil(P, M, d, p, m, ip, jp, kp, wx, wy, wz)) { report(err, DUSTB_ERR_POINT); return; }
  const double density = mass / (M.s(m, DX1) * M.s(m, DX2) * M.s(m, DX3));
  const double v1 = P.r(DUSTB_IPVX, p), v2 = P.r(DUSTB_IPVY, p), v3 = P.r(DUSTB_IPVZ, p);
  for (int c = 0; c < 3; ++c)
    for (int b = 0; b < 3; ++b)
      for (int a = 0; a < 3; ++a) {
        const double w = density * wz[c] * wy[b] * wx[a];
        if (w == 0.0) continue;
        const int kk = kp + c - 1, jj = jp + b - 1, ii = ip + a - 1;
        atomicAdd(&f[d.at(m, ncomp, 0, kk, jj, ii)], w);
        if (ncomp == 1) continue;
        atomicAdd(&f[d.at(m, ncomp, 1, kk, jj, ii)], w * v1);
        atomicAdd(&f[d.at(m, ncomp, 2, kk, jj, ii)], w * v2);
        atomicAdd(&f[d.at(m, ncomp, 3, kk, jj, ii)], w * v3);
      }
}

// the remapped field's active cells, the ghost cells zero (:246-248, :297-304)
__global__ void k_owned_copy(Ind d, const double *f, double *out, int nvar) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = d.cells();
  if (idx >= per * d.nmb * nvar) return;
  const long long mv = idx / per;
  long long r = idx - mv * per;
  const int i = (int)(r % d.n1); r /= d.n1;
  const int j = (int)(r % d.n2);
  const int k = (int)(r / d.n2);
  const bool act = i >= d.is && i <= d.ie && j >= d.js && j <= d.je && k >= d.ks && k <= d.ke;
  out[idx] = act ? f[idx] : 0.0;
}

// The transpose of the shear part of the deposit remap (shear_add_sum) for ghost cell
// (k, j, i) of face block m beyond the shear-periodic face in direction o1: the active cells
// its deposit lands in lie in the strip next to the opposite face, in the same x3 plane (or
// the neighbouring block's across an x3 ghost plane, or the mirrored plane at a physical x3
// face), in the global rows its interval [Y + sh, Y + 1 + sh) overlaps; the overlaps are the
// weights, formed as shear_add_sum forms them.
__device__ double shear_transpose_sum(const SBox &B, const Ind &d, const double *owned, int nvar,
                                      int m, int v, int k, int j, int i, int o1) {
  const int ng1 = B.ng - 1;
  const long long N2 = (long long)B.nb2 * B.nx2;
  int b2, b3;
  B.b23(m, b2, b3);
  const int g = (o1 > 0) ? i - d.ie - 1 : i - (d.is - d.ng);
  const int tface = (o1 > 0) ? 0 : 1;
  const int ti = (o1 > 0) ? d.is + g : d.ie - ng1 + g;
  const double sh = (o1 > 0) ? B.shR : -B.shR;
  int tb3 = b3, tk = k;
  if (k > d.ke) {
    if (b3 < B.nb3 - 1 || B.x3bc == 0) { tb3 = (b3 + 1) % B.nb3; tk = k - B.nx3; }
    else if (!B.drop) tk = 2 * d.ke + 1 - k;
    else return 0.0;
  } else if (k < d.ks) {
    if (b3 > 0 || B.x3bc == 0) { tb3 = (b3 + B.nb3 - 1) % B.nb3; tk = k + B.nx3; }
    else if (!B.drop) tk = 2 * d.ks - 1 - k;
    else return 0.0;
  }
  const long long Y = (long long)b2 * B.nx2 + (j - d.js);
  const double ya = (double)Y + sh, yb = (double)(Y + 1) + sh;
  const long long F = (long long)floor(ya);
  double sum = 0.0;
  for (long long Jg = F; Jg <= F + 1; ++Jg) {
    const double clo = (double)Jg, chi = clo + 1.0;
    const double o = fmin(yb, chi) - fmax(ya, clo);
    if (!(o > 0.0)) continue;
    const long long J = ((Jg % N2) + N2) % N2;
    const int tb2 = (int)(J / B.nx2);
    const int T = B.block(tface, tb3, tb2);
    if (T < 0) continue;
    const int tj = (int)(J - (long long)tb2 * B.nx2) + d.js;
    sum += o * owned[d.at(T, nvar, v, tk, tj, ti)];
  }
  return sum;
}

// GatherPointGravityAcceleration's force field (:325-337, with the transpose of the deposit
// remap, GatherMap :121-160): the owned values on the active cells, and in every ghost cell the
// owned values of the active cells a deposit into that ghost cell lands in, times the remap
// weight -- the same-level neighbour's cell, the mirrored cell behind a physical x3 face (of the
// block or of its x1/x2 neighbour), or the overlap-weighted cells across a shear-periodic face
__global__ void k_point_force_field(Ind d, const int *nghbr, int gids, SBox B,
                                    const double *owned, double *f, int nvar) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = d.cells();
  if (idx >= per * d.nmb) return;
  const int m = (int)(idx / per);
  long long r = idx - (long long)m * per;
  const int i = (int)(r % d.n1); r /= d.n1;
  const int j = (int)(r % d.n2);
  const int k = (int)(r / d.n2);
  const int o1 = (i < d.is) ? -1 : ((i > d.ie) ? 1 : 0);
  const int o2 = (j < d.js) ? -1 : ((j > d.je) ? 1 : 0);
  const int o3 = (k < d.ks) ? -1 : ((k > d.ke) ? 1 : 0);
  if ((o1 | o2 | o3) == 0) {
    for (int v = 0; v < nvar; ++v) f[d.at(m, nvar, v, k, j, i)] = owned[d.at(m, nvar, v, k, j, i)];
    return;
  }
  if (B.on && B.crossing(m, o1)) {
    for (int v = 0; v < nvar; ++v)
      f[d.at(m, nvar, v, k, j, i)] = shear_transpose_sum(B, d, owned, nvar, m, v, k, j, i, o1);
    return;
  }
  int src = -1, sk = k - o3 * d.nx3;
  if (o3 != 0 && nghbr[(long long)m * 27 + dir_slot(0, 0, o3)] < 0) {
    // behind a physical x3 face: the fold's mirrored plane, in this block or its x1/x2
    // neighbour (the deposit is never dropped here)
    src = (o1 | o2) ? nghbr[(long long)m * 27 + dir_slot(o1, o2, 0)] - gids : m;
    sk = (o3 < 0) ? 2 * d.ks - 1 - k : 2 * d.ke + 1 - k;
  } else {
    src = nghbr[(long long)m * 27 + dir_slot(o1, o2, o3)] - gids;
  }
  const bool ok = src >= 0 && src < d.nmb;
  for (int v = 0; v < nvar; ++v)
    f[d.at(m, nvar, v, k, j, i)] =
        ok ? owned[d.at(src, nvar, v, sk, j - o2 * d.nx2, i - o1 * d.nx1)] : 0.0;
}

// the acceleration at each particle: the TSC weights over the force field (:339-368)
__global__ void k_point_gather(PCtx P, MCtx M, Ind d, const double *f, double *acc,
                               long long astride, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  double a[3] = {0.0, 0.0, 0.0};
  const double mass = P.r(DUSTB_IPM, p);
  int m, ip, jp, kp; double wx[3], wy[3], wz[3];
  if (!(mass >= 0.0) || !isfinite(mass)) {
    report(err, DUSTB_ERR_POINT);
  } else if (mass != 0.0) {
    if (!point_stencil(P, M, d, p, m, ip, jp, kp, wx, wy, wz)) {
      report(err, DUSTB_ERR_POINT);
    } else {
      for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 3; ++b)
          for (int q = 0; q < 3; ++q) {
            const double w = wz[c] * wy[b] * wx[q];
            for (int v = 0; v < 3; ++v)
              a[v] += w * f[d.at(m, 3, v, kp + c - 1, jp + b - 1, ip + q - 1)];
          }
      if (!isfinite(a[0]) || !isfinite(a[1]) || !isfinite(a[2])) report(err, DUSTB_ERR_POINT);
    }
  }
  for (int v = 0; v < 3; ++v) acc[(long long)v * astride + p] = a[v];
}

// ---- refinable clouds on a uniform mesh: plain P1 hat clouds ------------------------------
// CloudShape1D (src/dust/dust.hpp:240-298; HatCDF / HatMoment :169-182) for a cloud without
// lobes: along each direction the hat of half-width ell = dx / 2^level about the particle, a
// cell's weight the difference of the hat CDF at its faces, its first moment about the
// particle ell times the difference of the moment antiderivative.  LeafTraversal3D::ForEach
// (src/dust/dust_leaf3d.hpp:368-513) on a uniform mesh: the cells of the block and of its
// same-level neighbours under the support, each cell's faces from its own block's origin (the
// neighbour's periodic image next to the block); across a physical x3 face a second part, the
// cloud mirrored about the face, whose x3 moments are taken about the particle; leaves in the
// order part, z, y, x (lower neighbour, block, upper neighbour along each), zero-weight leaves
// skipped.  2-D (LeafTraversal::ForEach): no x3 direction.
__device__ __forceinline__ double hat_cdf(double s) {
  if (s <= -1.0) return 0.0;
  if (s >= 1.0) return 1.0;
  return (s <= 0.0) ? 0.5 * (1.0 + s) * (1.0 + s) : 1.0 - 0.5 * (1.0 - s) * (1.0 - s);
}
__device__ __forceinline__ double hat_moment(double s) {
  if (s <= -1.0 || s >= 1.0) return 1.0 / 6.0;
  return (s <= 0.0) ? 0.5 * (s * s) + (s * s) * s / 3.0 : 0.5 * (s * s) - (s * s) * s / 3.0;
}

// cloud code bits (CloudGeometry, src/dust/dust.hpp:101-125)
constexpr int kCodeLevel = 15, kCodeLobe2 = 4, kCodeLobe1 = 6, kCodeLobe3 = 9;
constexpr int kCodeBits = 15 | (3 << 4) | (3 << 6) | (3 << 9);

struct CloudAxis {
  int n;
  int o[6], i[6];
  double w[6], g[6], org[6];   // weight, moment, the origin of the cell's block image
};

__device__ void cloud_axis(const MCtx &M, const Ind &d, int m, int a, double x, int lev,
                           double L, CloudAxis &A) {
  const int nx = (a == 0) ? d.nx1 : ((a == 1) ? d.nx2 : d.nx3);
  const double dx = M.s(m, DX1 + a), idx = 1.0 / dx;
  const double ell = ldexp(dx, -lev), inv = ldexp(idx, lev);
  const double lo = x - ell, hi = x + ell;
  A.n = 0;
  for (int o = -1; o <= 1; ++o) {
    int b = m;
    if (o != 0) {
      const int gid = M.nghbr[(long long)m * 27 + dir_slot(a == 0 ? o : 0, a == 1 ? o : 0,
                                                           a == 2 ? o : 0)];
      if (gid < 0 || gid - M.gids < 0 || gid - M.gids >= d.nmb) continue;
      b = gid - M.gids;
    }
    double bx0 = M.s(b, X1MIN + a);
    if (o < 0 && M.s(b, X1MIN + a) >= M.s(m, X1MIN + a)) bx0 -= L;
    if (o > 0 && M.s(b, X1MIN + a) <= M.s(m, X1MIN + a)) bx0 += L;
    int i0 = (int)floor((lo - bx0) * idx), i1 = (int)ceil((hi - bx0) * idx) - 1;
    i0 = (i0 < 0) ? 0 : i0;
    i1 = (i1 > nx - 1) ? nx - 1 : i1;
    for (int i = i0; i <= i1 && A.n < 6; ++i) {
      const double za = (bx0 + i * dx - x) * inv, zb = (bx0 + (i + 1) * dx - x) * inv;
      A.o[A.n] = o; A.i[A.n] = i; A.org[A.n] = bx0;
      A.w[A.n] = hat_cdf(zb) - hat_cdf(za);
      A.g[A.n] = ell * (hat_moment(zb) - hat_moment(za));
      ++A.n;
    }
  }
}

// the position of a cloud in the frame of block m; true if this build takes it: a level code
// without lobe bits, a position inside the block (slack: within that many cells of it)
__device__ bool cloud_frame_ok(const MCtx &M, const Ind &d, int m, int lev, const double L[3],
                               double x[3], double slack) {
  if (!block_ok(d, m) || (lev & ~(M.lt.on ? kCodeBits : kCodeLevel)) != 0) return false;
  const int nx[3] = {d.nx1, d.nx2, d.nx3};
  for (int a = 0; a < (d.three_d ? 3 : 2); ++a) {
    const double cx = M.s(m, X1MIN + a) + 0.5 * nx[a] * M.s(m, DX1 + a);
    x[a] -= L[a] * round((x[a] - cx) * (1.0 / L[a]));
    const double e = slack * M.s(m, DX1 + a);
    if (!(x[a] >= M.s(m, X1MIN + a) - e && x[a] < M.s(m, X1MAX + a) + e)) return false;
  }
  return true;
}

// the stage position (3-D: y + sh x, the gas in its orbital-advection frame; 2-D: no shift)
__device__ bool cloud_load(const PCtx &P, const MCtx &M, const Ind &d, int p, double sh,
                           const double L[3], int &m, double x[3], int &lev) {
  m = P.i(DUSTB_PGID, p) - M.gids;
  lev = P.i(DUSTB_PLEV, p);
  x[0] = P.r(DUSTB_IPX, p);
  x[1] = d.three_d ? P.r(DUSTB_IPY, p) + sh * P.r(DUSTB_IPX, p) : P.r(DUSTB_IPY, p);
  x[2] = d.three_d ? P.r(DUSTB_IPZ, p) : 0.0;
  return cloud_frame_ok(M, d, m, lev, L, x, 0.0);
}

__device__ __forceinline__ int cloud_owner(const MCtx &M, const Ind &d, int m, int ox, int oy,
                                           int oz) {
  if (!ox && !oy && !oz) return m;
  const int gid = M.nghbr[(long long)m * 27 + dir_slot(ox, oy, oz)];
  const int b = gid - M.gids;
  return (gid < 0 || b < 0 || b >= d.nmb) ? -1 : b;
}

// the cell measure: the volume, 2-D the area (LeafApi::Measure)
__device__ __forceinline__ double cloud_measure(const MCtx &M, const Ind &d, int b) {
  return d.three_d ? M.s(b, DX1) * M.s(b, DX2) * M.s(b, DX3) : M.s(b, DX1) * M.s(b, DX2);
}

struct CloudLeaf {
  int b, k, j, i;              // owner block, padded cell
  double w, m1x, m1y, m1z;
};

// ---- refinable clouds on a refined 3-D mesh: the leaf traversal -------------------------
// LeafTraversal3D (src/dust/dust_leaf3d.hpp), one rank, no shear: a cloud anchored at block m
// is integrated over the leaf cells of every block its support meets, each cell's weight the
// product of the three 1-D integrals of the cloud shape (CloudShape1D with transition lobes,
// src/dust/dust.hpp:240-298) between the cell's faces.  Candidates: m alone when the support
// lies inside it; m and its distinct neighbours when the safe ring or the band scan shows they
// cover the support (NeedGlobal / Covered); otherwise every block and periodic image that
// meets it.  Leaves in the order part, candidate, runs of 4 cells in x, z, y, x.


struct Shape1 {
  double x, ell, inv, sl, lo, hi;
  int lobe;
  bool both, point;
};
__device__ __forceinline__ Shape1 make_shape(double x, double ell_in, double inv_in,
                                             int lobe_in, bool point) {
  Shape1 s;
  s.both = (lobe_in == 3);
  s.ell = s.both ? 2.0 * ell_in : ell_in;
  s.lobe = s.both ? 0 : lobe_in;
  s.sl = (s.lobe == 1) ? -s.ell : s.ell;
  s.lo = (s.lobe == 1) ? x - 2.0 * s.ell : x - s.ell;
  s.hi = (s.lobe == 2) ? x + 2.0 * s.ell : x + s.ell;
  s.x = x;
  s.point = point;
  s.inv = s.both ? 0.5 * inv_in : inv_in;
  return s;
}
struct Face1 { double c, cl, h, hl; };
template <bool kM>
__device__ __forceinline__ Face1 face_at(const Shape1 &s, double z) {
  Face1 f{0.0, 0.0, 0.0, 0.0};
  const double sz = (z - s.x) * s.inv;
  f.c = hat_cdf(sz);
  if (kM) f.h = hat_moment(sz);
  if (s.lobe) {
    const double tz = (z - s.x - s.sl) * s.inv;
    f.cl = hat_cdf(tz);
    if (kM) f.hl = hat_moment(tz);
  }
  return f;
}
template <bool kM>
__device__ __forceinline__ void cell_1d(const Shape1 &s, const Face1 &a, const Face1 &b,
                                        double &w, double &g) {
  w = b.c - a.c;
  g = 0.0;
  if (kM) g = (s.both && s.point) ? 0.0 : s.ell * (b.h - a.h);
  if (s.lobe) {
    const double wl = b.cl - a.cl;
    w = (2.0 / 3.0) * w + (1.0 / 3.0) * wl;
    if (kM) g = s.point ? 0.0 : (2.0 / 3.0) * g + (1.0 / 3.0) * (s.ell * (b.hl - a.hl) + s.sl * wl);
  }
}

__device__ __forceinline__ int floor_div(int a, int n) {
  int q = a / n;
  if ((a % n != 0) && ((a < 0) != (n < 0))) --q;
  return q;
}
// the periodic images k0..k1 of [c0 - r, c1 + r) that meet [a, b] (LeafTraversal::ImageRange)
__device__ __forceinline__ void image_range(int c0, int c1, int r, int n, int a, int b, int &k0,
                                            int &k1) {
  k0 = floor_div(a - (c1 + r), n) + 1;
  k1 = floor_div(b - (c0 - r), n);
}

// ForCandidates (src/dust/dust_leaf3d.hpp:142-180): f(b, sx, sy, sz), block b moved by
// -(sx, sy, sz) domain lengths; local: m, then its neighbours; global: every block's images
// that meet the finest-cell box [ia, ib] x [ja, jb] x [ka, kb] widened by r.  f returns false
// to stop.
template <typename F>
__device__ void for_candidates(const LTab &T, int m, bool global, int ia, int ib, int ja,
                               int jb, int ka, int kb, int r, F &&f) {
  if (!global) {
    if (!f(m, 0, 0, 0)) return;
    const int n = T.nnb[m];
    for (int k = 0; k < n; ++k) {
      const int *s = T.nbs + ((long long)m * DUSTB_LEAF_MAXNB + k) * 3;
      if (!f(T.nb[(long long)m * DUSTB_LEAF_MAXNB + k], s[0], s[1], s[2])) return;
    }
    return;
  }
  for (int b = 0; b < T.nmb; ++b) {
    const int *fb = T.fbox + 6 * (long long)b;
    int kx0, kx1, ky0, ky1, kz0, kz1;
    image_range(fb[0], fb[1], r, T.nf[0], ia, ib, kx0, kx1);
    image_range(fb[2], fb[3], r, T.nf[1], ja, jb, ky0, ky1);
    image_range(fb[4], fb[5], r, T.nf[2], ka, kb, kz0, kz1);
    if (!T.x3per) {
      if (kz0 > 0 || kz1 < 0) continue;
      kz0 = 0; kz1 = 0;
    }
    for (int kz = kz0; kz <= kz1; ++kz)
      for (int ky = ky0; ky <= ky1; ++ky)
        for (int kx = kx0; kx <= kx1; ++kx)
          if (!f(b, -kx, -ky, -kz)) return;
  }
}
// the finest-cell box of block b's image (sx, sy, sz) widened by r: [x0, x1) ...
__device__ __forceinline__ void image_rect(const LTab &T, int b, int sx, int sy, int sz, int r,
                                           int q[6]) {
  const int *fb = T.fbox + 6 * (long long)b;
  q[0] = fb[0] - sx * T.nf[0] - r; q[1] = fb[1] - sx * T.nf[0] + r;
  q[2] = fb[2] - sy * T.nf[1] - r; q[3] = fb[3] - sy * T.nf[1] + r;
  q[4] = fb[4] - sz * T.nf[2] - r; q[5] = fb[5] - sz * T.nf[2] + r;
}
// Meets (:181-197): a candidate of level >= minlev, widened by r, meets the box
__device__ bool leaf_meets(const LTab &T, int m, int ia, int ib, int ja, int jb, int ka, int kb,
                           int minlev, int r, bool global) {
  bool hit = false;
  for_candidates(T, m, global, ia, ib, ja, jb, ka, kb, r, [&](int b, int sx, int sy, int sz) {
    if (T.blev[b] < minlev) return true;
    int q[6];
    image_rect(T, b, sx, sy, sz, r, q);
    if (ib < q[0] || ia >= q[1] || jb < q[2] || ja >= q[3] || kb < q[4] || ka >= q[5]) return true;
    hit = true;
    return false;
  });
  return hit;
}
// Covered (:198-238): the band scan, slab by slab in z; every box taken holds the cell it was
// taken for
__device__ bool leaf_covered(const LTab &T, int m, int ia, int ib, int ja, int jb, int ka, int kb,
                             int minlev, int r, bool global) {
  int z = ka;
  while (z <= kb) {
    int ztop = kb + 1;
    int y = ja;
    while (y <= jb) {
      int x = ia, top = jb + 1;
      while (x <= ib) {
        int xe = x, ye = y, ze = z;
        for_candidates(T, m, global, x, x, y, y, z, z, r, [&](int b, int sx, int sy, int sz) {
          if (T.blev[b] < minlev) return true;
          int q[6];
          image_rect(T, b, sx, sy, sz, r, q);
          if (x < q[0] || x >= q[1] || y < q[2] || y >= q[3] || z < q[4] || z >= q[5]) return true;
          if (q[1] > xe || (q[1] == xe && q[3] > ye) || (q[1] == xe && q[3] == ye && q[5] > ze)) {
            xe = q[1]; ye = q[3]; ze = q[5];
          }
          return true;
        });
        if (xe == x) return false;
        top = (ye < top) ? ye : top;
        ztop = (ze < ztop) ? ze : ztop;
        x = xe;
      }
      y = top;
    }
    z = ztop;
  }
  return true;
}
__device__ __forceinline__ void clip_z(const LTab &T, int &ka, int &kb) {
  if (T.x3per) return;
  ka = (ka < 0) ? 0 : ka;
  kb = (kb > T.nf[2] - 1) ? T.nf[2] - 1 : kb;
}
// NeedGlobal (:253-272): the box widened by r is not inside the safe ring of m nor covered by m
// and its neighbours
__device__ bool leaf_need_global(const LTab &T, int m, int ia, int ib, int ja, int jb, int ka,
                                 int kb, int r) {
  const int a1 = ia - r, b1 = ib + r;
  int c1 = ka - r, d1 = kb + r;
  clip_z(T, c1, d1);
  int q[6];
  image_rect(T, m, 0, 0, 0, 0, q);
  const int *sf = T.safe + 3 * (long long)m;
  if (q[0] - sf[0] <= a1 && q[1] + sf[0] > b1 && q[2] - sf[1] <= ja - r && q[3] + sf[1] > jb + r &&
      q[4] - sf[2] <= c1 && q[5] + sf[2] > d1)
    return false;
  return !leaf_covered(T, m, a1, b1, ja - r, jb + r, c1, d1, 0, 0, false);
}

// ForEach (:368-513) without shear: f(leaf) for every leaf under the cloud `code` at the framed
// position x (anchor m); kM: the moment traversal of the gathers (GatherCode: the point rule
// along lobed directions)
template <bool kM, typename F>
__device__ void leaf_foreach(const MCtx &M, const Ind &d, int m, const double x[3], int code,
                             F &&f) {
  const LTab &T = M.lt;
  const double Lz = M.x3max - M.x3min;
  const int lev = code & kCodeLevel;
  const int lb1 = (code >> kCodeLobe1) & 3, lb2 = (code >> kCodeLobe2) & 3;
  const int lb3 = (code >> kCodeLobe3) & 3;
  const bool point = kM;
  const double h1 = ldexp(T.rdx[0], -lev), ih1 = ldexp(T.irdx[0], lev);
  const double h2 = ldexp(T.rdx[1], -lev), ih2 = ldexp(T.irdx[1], lev);
  const double h3 = ldexp(T.rdx[2], -lev), ih3 = ldexp(T.irdx[2], lev);
  const Shape1 s1 = make_shape(x[0], h1, ih1, lb1, point);
  const Shape1 s2 = make_shape(x[1], h2, ih2, lb2, point);
  Shape1 s3 = make_shape(x[2], h3, ih3, lb3, point);
  int npz = 1, zside = 0;
  if (!T.x3per && (s3.lo < M.x3min || s3.hi > M.x3max)) { npz = 2; zside = (s3.hi > M.x3max) ? 1 : 0; }
  const double Lx = M.x1max - M.x1min, Ly = M.x2max - M.x2min;
#pragma unroll 1
  for (int part = 0; part < npz; ++part) {
    double zp = x[2];
    if (part == 1) {
      zp = 2.0 * ((zside == 1) ? M.x3max : M.x3min) - x[2];
      s3 = make_shape(zp, h3, ih3, (lb3 == 1 || lb3 == 2) ? 3 - lb3 : lb3, point);
    }
    const bool zcorr = kM && part == 1;
    const double ax0 = M.s(m, X1MIN), ay0 = M.s(m, X2MIN), az0 = M.s(m, X3MIN);
    const bool inside = s1.lo >= ax0 && s1.hi <= ax0 + d.nx1 * M.s(m, DX1) && s2.lo >= ay0 &&
                        s2.hi <= ay0 + d.nx2 * M.s(m, DX2) && s3.lo >= az0 &&
                        s3.hi <= az0 + d.nx3 * M.s(m, DX3);
    // one candidate: its cells under the support
    auto visit = [&](int b, int sx, int sy, int sz) {
      const double dx = M.s(b, DX1), dy = M.s(b, DX2), dz = M.s(b, DX3);
      const double bx0 = M.s(b, X1MIN) - sx * Lx, by0 = M.s(b, X2MIN) - sy * Ly;
      const double bz0 = M.s(b, X3MIN) - sz * Lz;
      const double idx = 1.0 / dx, idy = 1.0 / dy, idz = 1.0 / dz;
      int i0 = (int)floor((s1.lo - bx0) * idx), i1 = (int)ceil((s1.hi - bx0) * idx) - 1;
      int j0 = (int)floor((s2.lo - by0) * idy), j1 = (int)ceil((s2.hi - by0) * idy) - 1;
      int k0 = (int)floor((s3.lo - bz0) * idz), k1 = (int)ceil((s3.hi - bz0) * idz) - 1;
      i0 = (i0 < 0) ? 0 : i0; i1 = (i1 > d.nx1 - 1) ? d.nx1 - 1 : i1;
      j0 = (j0 < 0) ? 0 : j0; j1 = (j1 > d.nx2 - 1) ? d.nx2 - 1 : j1;
      k0 = (k0 < 0) ? 0 : k0; k1 = (k1 > d.nx3 - 1) ? d.nx3 - 1 : k1;
#pragma unroll 1
      for (int ic = i0; ic <= i1; ic += 4) {
        const int nr = (i1 - ic + 1 < 4) ? i1 - ic + 1 : 4;
        double w1[4], g1[4];
        Face1 f1 = face_at<kM>(s1, bx0 + ic * dx);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          w1[a] = 0.0; g1[a] = 0.0;
          if (a < nr) {
            const Face1 fn = face_at<kM>(s1, bx0 + (ic + a + 1) * dx);
            cell_1d<kM>(s1, f1, fn, w1[a], g1[a]);
            f1 = fn;
          }
        }
        Face1 f3 = face_at<kM>(s3, bz0 + k0 * dz);
#pragma unroll 1
        for (int k = k0; k <= k1; ++k) {
          const Face1 fn3 = face_at<kM>(s3, bz0 + (k + 1) * dz);
          double w3, g3;
          cell_1d<kM>(s3, f3, fn3, w3, g3);
          f3 = fn3;
          if (w3 == 0.0 && (!kM || g3 == 0.0)) continue;
          double czk = 0.0;
          if (zcorr) {
            const double zc = bz0 + (k + 0.5) * dz;
            const double e = x[2] - zc;
            czk = (zp - zc) - (e - Lz * round(e / Lz));
          }
          Face1 f2 = face_at<kM>(s2, by0 + j0 * dy);
#pragma unroll 1
          for (int j = j0; j <= j1; ++j) {
            const Face1 fn2 = face_at<kM>(s2, by0 + (j + 1) * dy);
            double w2, g2;
            cell_1d<kM>(s2, f2, fn2, w2, g2);
            f2 = fn2;
            if (w2 == 0.0 && (!kM || g2 == 0.0)) continue;
            const double w23 = w2 * w3;
#pragma unroll 1
            for (int a = 0; a < nr; ++a) {
              CloudLeaf lf;
              lf.w = w23 * w1[a];
              lf.m1x = lf.m1y = lf.m1z = 0.0;
              if (kM) {
                lf.m1x = w23 * g1[a];
                lf.m1y = w1[a] * g2 * w3;
                lf.m1z = w1[a] * w2 * g3;
                if (zcorr) lf.m1z += czk * lf.w;
                if (lf.w == 0.0 && lf.m1x == 0.0 && lf.m1y == 0.0 && lf.m1z == 0.0) continue;
              } else if (lf.w == 0.0) {
                continue;
              }
              lf.b = b; lf.k = d.ks + k; lf.j = d.js + j; lf.i = d.is + ic + a;
              f(lf);
            }
          }
        }
      }
    };
    // Candidates (:319-366): the support's finest-cell box (not needed when it lies inside m)
    bool global = false;
    int box[6] = {0, 0, 0, 0, 0, 0};
    if (!inside) {
      box[0] = (int)floor((s1.lo - M.x1min) / T.fdx[0]);
      box[1] = (int)ceil((s1.hi - M.x1min) / T.fdx[0]) - 1;
      box[2] = (int)floor((s2.lo - M.x2min) / T.fdx[1]);
      box[3] = (int)ceil((s2.hi - M.x2min) / T.fdx[1]) - 1;
      box[4] = (int)floor((s3.lo - M.x3min) / T.fdx[2]);
      box[5] = (int)ceil((s3.hi - M.x3min) / T.fdx[2]) - 1;
      clip_z(T, box[4], box[5]);
      global = leaf_need_global(T, m, box[0], box[1], box[2], box[3], box[4], box[5], 0);
    }
    // one loop over the candidates in ForCandidates' order with a single visit: m alone when
    // inside; m then its neighbours (local); every block and its periodic images meeting the box
    // widened by one finest cell (global); each taken only when its box meets the support.
    // (One call site keeps the kernel's code small: two made it stall on instruction fetch.)
    const int nloc = inside ? 0 : T.nnb[m];
    int c = global ? 0 : -1;                       // local: -1 is m; global: the next block
    int cur = 0, img = 0, nimg = 0, kx0 = 0, nx = 1, ky0 = 0, ny = 1, kz0 = 0;
#pragma unroll 1
    while (true) {
      int b, sx, sy, sz;
      if (!global) {
        if (c >= nloc) break;
        if (c < 0) {
          b = m; sx = sy = sz = 0;
        } else {
          const int *sh = T.nbs + ((long long)m * DUSTB_LEAF_MAXNB + c) * 3;
          b = T.nb[(long long)m * DUSTB_LEAF_MAXNB + c]; sx = sh[0]; sy = sh[1]; sz = sh[2];
        }
        ++c;
      } else {
        if (img >= nimg) {
          if (c >= T.nmb) break;
          const int *fb = T.fbox + 6 * (long long)c;
          int kx1, ky1, kz1, kz0_;
          image_range(fb[0], fb[1], 0, T.nf[0], box[0] - 1, box[1] + 1, kx0, kx1);
          image_range(fb[2], fb[3], 0, T.nf[1], box[2] - 1, box[3] + 1, ky0, ky1);
          image_range(fb[4], fb[5], 0, T.nf[2], box[4] - 1, box[5] + 1, kz0_, kz1);
          kz0 = kz0_;
          if (!T.x3per) {
            if (kz0 > 0 || kz1 < 0) { kz0 = 0; kz1 = -1; } else { kz0 = 0; kz1 = 0; }
          }
          nx = kx1 - kx0 + 1; ny = ky1 - ky0 + 1;
          const int nz = kz1 - kz0 + 1;
          nimg = (nx > 0 && ny > 0 && nz > 0) ? nx * ny * nz : 0;
          img = 0;
          cur = c++;
          continue;
        }
        // images in the order kz, ky, kx (kx fastest)
        b = cur;
        sx = -(kx0 + img % nx);
        sy = -(ky0 + (img / nx) % ny);
        sz = -(kz0 + img / (nx * ny));
        ++img;
      }
      bool take = inside;
      if (!take) {
        const double bx0 = M.s(b, X1MIN) - sx * Lx, by0 = M.s(b, X2MIN) - sy * Ly;
        const double bz0 = M.s(b, X3MIN) - sz * Lz;
        take = !(s1.hi <= bx0 || s1.lo >= bx0 + d.nx1 * M.s(b, DX1) || s2.hi <= by0 ||
                 s2.lo >= by0 + d.nx2 * M.s(b, DX2) || s3.hi <= bz0 ||
                 s3.lo >= bz0 + d.nx3 * M.s(b, DX3));
      }
      if (take) visit(b, sx, sy, sz);
    }
  }
}

// ---- the owner leaf, the instant switch and the P1 split ----------------------------------
// the periodic image of a point next to block m (LeafTraversal3D::Frame without shear)
__device__ __forceinline__ void leaf_frame(const MCtx &M, const Ind &d, int m, double x[3]) {
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  const int nx[3] = {d.nx1, d.nx2, d.nx3};
  for (int a = 0; a < 3; ++a) {
    if (a == 2 && !M.lt.x3per) break;
    const double c = M.s(m, X1MIN + a) + 0.5 * nx[a] * M.s(m, DX1 + a);
    x[a] -= L[a] * round((x[a] - c) * (1.0 / L[a]));
  }
}
// Locate (:515-533): the block holding the finest cell (ic, jc, kc), -1 if none
__device__ int leaf_locate(const LTab &T, const Ind &d, int ic, int jc, int kc) {
  ic = ((ic % T.nf[0]) + T.nf[0]) % T.nf[0];
  jc = ((jc % T.nf[1]) + T.nf[1]) % T.nf[1];
  if (!T.x3per && (kc < 0 || kc >= T.nf[2])) return -1;
  kc = ((kc % T.nf[2]) + T.nf[2]) % T.nf[2];
  for (int l = 0; l <= T.nlev; ++l) {
    const int sh = T.nlev - l;
    const long long key = ((long long)l << 57) | ((long long)(kc / (d.nx3 << sh)) << 38) |
                          ((long long)(jc / (d.nx2 << sh)) << 19) | (long long)(ic / (d.nx1 << sh));
    int lo = 0, hi = T.nmb;
    while (lo < hi) {
      const int mid = (lo + hi) / 2;
      if (T.lockey[mid] < key) lo = mid + 1; else hi = mid;
    }
    if (lo < T.nmb && T.lockey[lo] == key) return T.locblk[lo];
  }
  return -1;
}
// Owner (:534-595) without shear: the block whose leaf holds the point, searched from block m
// (m and its neighbours, then the location index); -1 if none
__device__ int leaf_owner(const MCtx &M, const Ind &d, const double px[3], int m) {
  const LTab &T = M.lt;
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  double x[3] = {px[0], px[1], px[2]};
  leaf_frame(M, d, m, x);
  if (!T.x3per) {
    if (x[2] < M.x3min) x[2] = 2.0 * M.x3min - x[2];
    if (x[2] >= M.x3max) x[2] = fmin(2.0 * M.x3max - x[2], M.x3max - 1.0e-12 * L[2]);
  }
  const int ic = (int)floor((x[0] - M.x1min) / T.fdx[0]);
  const int jc = (int)floor((x[1] - M.x2min) / T.fdx[1]);
  const int kc = (int)floor((x[2] - M.x3min) / T.fdx[2]);
  int res = -1;
  for_candidates(T, m, false, 0, 0, 0, 0, 0, 0, 0, [&](int b, int sx, int sy, int sz) {
    const double fi = (x[0] - (M.s(b, X1MIN) - sx * L[0])) / M.s(b, DX1);
    const double fj = (x[1] - (M.s(b, X2MIN) - sy * L[1])) / M.s(b, DX2);
    const double fk = (x[2] - (M.s(b, X3MIN) - sz * L[2])) / M.s(b, DX3);
    if (!(fi >= 0.0 && fi < d.nx1 && fj >= 0.0 && fj < d.nx2 && fk >= 0.0 && fk < d.nx3))
      return true;
    res = b;
    return false;
  });
  return (res >= 0) ? res : leaf_locate(T, d, ic, jc, kc);
}

__device__ __forceinline__ int leaf_anchor(const MCtx &M, const Ind &d, int pgid) {
  const int m = pgid - M.gids;
  return (m >= 0 && m < d.nmb) ? m : 0;
}

// CloudInstantSwitch's kernel (InstantSwitchLevels, src/dust/dust_cloud.cpp:1023-1045)
__global__ void k_cloud_instant_switch(PCtx P, MCtx M, Ind d, int L, int *nchange) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const int code = P.i(DUSTB_PLEV, p);
  if ((code & ~kCodeLevel) != 0 || code < L) return;
  const double x[3] = {P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p), P.r(DUSTB_IPZ, p)};
  const int b = leaf_owner(M, d, x, leaf_anchor(M, d, P.i(DUSTB_PGID, p)));
  if (b < 0) return;
  const int lev = (M.lt.blev[b] > L) ? M.lt.blev[b] : L;
  if (lev != code) {
    P.i(DUSTB_PLEV, p) = lev;
    atomicAdd(nchange, 1);
  }
}

struct SplitCtl {
  int max_level, everywhere, overlap;
  int rdil[18];
  double slack;
};

// AnyAbove / AllAbove (:596-622): a leaf above lev meets (all) or covers the box
__device__ bool leaf_above(const LTab &T, const SplitCtl &C, int m, int ia, int ib, int ja,
                           int jb, int ka, int kb, int lev, bool all) {
  if (lev + 1 > T.nlev) return false;
  const int r = C.rdil[lev + 1];
  const bool g = leaf_need_global(T, m, ia, ib, ja, jb, ka, kb, r);
  if (!g && m < T.nmb && lev + 1 > T.nbmax[m] && ia <= ib && ja <= jb && ka <= kb) return false;
  return all ? leaf_covered(T, m, ia, ib, ja, jb, ka, kb, lev + 1, r, g)
             : leaf_meets(T, m, ia, ib, ja, jb, ka, kb, lev + 1, r, g);
}
// InsideFiner (:668-681) with SupportBox (:653-666): the plain level-lev cloud's support, shrunk
// by the slack, meets (split_overlap) or lies on leaves finer than lev
__device__ bool leaf_inside_finer(const MCtx &M, const Ind &d, const SplitCtl &C, double px,
                                  double py, double pz, int lev, int m) {
  const LTab &T = M.lt;
  if (lev >= T.nlev || lev >= C.max_level) return false;
  if (C.everywhere) return true;
  double x[3] = {px, py, pz};
  leaf_frame(M, d, m, x);
  const double f = 1.0 - C.slack;
  const double r1 = f * T.rdx[0] / (double)(1 << lev), r2 = f * T.rdx[1] / (double)(1 << lev);
  const double r3 = f * T.rdx[2] / (double)(1 << lev);
  const int ia = (int)floor((x[0] - r1 - M.x1min) / T.fdx[0]);
  const int ib = (int)ceil((x[0] + r1 - M.x1min) / T.fdx[0]) - 1;
  const int ja = (int)floor((x[1] - r2 - M.x2min) / T.fdx[1]);
  const int jb = (int)ceil((x[1] + r2 - M.x2min) / T.fdx[1]) - 1;
  int ka = (int)floor((x[2] - r3 - M.x3min) / T.fdx[2]);
  int kb = (int)ceil((x[2] + r3 - M.x3min) / T.fdx[2]) - 1;
  clip_z(T, ka, kb);
  return leaf_above(T, C, m, ia, ib, ja, jb, ka, kb, lev, !C.overlap);
}
__device__ __forceinline__ double half_width(const LTab &T, int lev, int a) {
  return T.rdx[a] / (double)(1 << (lev & kCodeLevel));
}
// P1FlagT (src/dust/dust_cloud3d.cpp:188-210): is the cloud split (or a lobe released) now?
__device__ bool p1_flag(const MCtx &M, const Ind &d, const SplitCtl &C, int m, int code,
                        const double x[3]) {
  const int lev = code & kCodeLevel;
  const int l1 = (code >> kCodeLobe1) & 3, l2 = (code >> kCodeLobe2) & 3;
  const int l3 = (code >> kCodeLobe3) & 3;
  if (l1 == 0 && l2 == 0 && l3 == 0) return leaf_inside_finer(M, d, C, x[0], x[1], x[2], lev, m);
  if (lev > 0 && leaf_inside_finer(M, d, C, x[0], x[1], x[2], lev - 1, m)) {
    const double h1 = half_width(M.lt, lev - 1, 0), h2 = half_width(M.lt, lev - 1, 1);
    const double h3 = half_width(M.lt, lev - 1, 2);
    return ((l1 & 1) && leaf_inside_finer(M, d, C, x[0] - h1, x[1], x[2], lev - 1, m)) ||
           ((l1 & 2) && leaf_inside_finer(M, d, C, x[0] + h1, x[1], x[2], lev - 1, m)) ||
           ((l2 & 1) && leaf_inside_finer(M, d, C, x[0], x[1] - h2, x[2], lev - 1, m)) ||
           ((l2 & 2) && leaf_inside_finer(M, d, C, x[0], x[1] + h2, x[2], lev - 1, m)) ||
           ((l3 & 1) && leaf_inside_finer(M, d, C, x[0], x[1], x[2] - h3, lev - 1, m)) ||
           ((l3 & 2) && leaf_inside_finer(M, d, C, x[0], x[1], x[2] + h3, lev - 1, m));
  }
  return false;
}
// P1SepT (:229-250): bit 2a (2a + 1) when the lower (upper) side along a lies on finer leaves
__device__ int p1_sep(const MCtx &M, const Ind &d, const SplitCtl &C, int m, int code,
                      const double x[3]) {
  const int lev = code & kCodeLevel;
  const bool plain = (code & ~kCodeLevel) == 0;
  const int l = plain ? lev : lev - 1;
  const double h1 = half_width(M.lt, l, 0), h2 = half_width(M.lt, l, 1);
  const double h3 = half_width(M.lt, l, 2);
  return (leaf_inside_finer(M, d, C, x[0] - h1, x[1], x[2], l, m) ? 1 : 0) |
         (leaf_inside_finer(M, d, C, x[0] + h1, x[1], x[2], l, m) ? 2 : 0) |
         (leaf_inside_finer(M, d, C, x[0], x[1] - h2, x[2], l, m) ? 4 : 0) |
         (leaf_inside_finer(M, d, C, x[0], x[1] + h2, x[2], l, m) ? 8 : 0) |
         (leaf_inside_finer(M, d, C, x[0], x[1], x[2] - h3, l, m) ? 16 : 0) |
         (leaf_inside_finer(M, d, C, x[0], x[1], x[2] + h3, l, m) ? 32 : 0);
}
struct Piece { double off, frac; int lobe; };
// P1Pieces3 (:52-65): the pieces of a cloud along one direction
__device__ __forceinline__ int p1_pieces(int lobe_old, bool sep_lo, bool sep_hi, Piece out[3]) {
  int n = 0;
  const double total = 0.5 + 0.25 * ((lobe_old & 1) ? 1 : 0) + 0.25 * ((lobe_old & 2) ? 1 : 0);
  const bool lo = (lobe_old & 1) && sep_lo, hi = (lobe_old & 2) && sep_hi;
  const int lobe_new = lobe_old & ~((lo ? 1 : 0) | (hi ? 2 : 0));
  const double keep = 0.5 + 0.25 * ((lobe_new & 1) ? 1 : 0) + 0.25 * ((lobe_new & 2) ? 1 : 0);
  out[n].off = 0.0; out[n].frac = keep / total; out[n].lobe = lobe_new; ++n;
  if (lo) { out[n].off = -1.0; out[n].frac = 0.25 / total; out[n].lobe = 0; ++n; }
  if (hi) { out[n].off = 1.0; out[n].frac = 0.25 / total; out[n].lobe = 0; ++n; }
  return n;
}
// P1BuildT<3> (:268-281)
__device__ __forceinline__ void p1_build(int code, int sep, Piece pc[3][3], int n[3], int &clev) {
  const int lev = code & kCodeLevel;
  const int l1 = (code >> kCodeLobe1) & 3, l2 = (code >> kCodeLobe2) & 3;
  const int l3 = (code >> kCodeLobe3) & 3;
  const bool plain = (l1 == 0 && l2 == 0 && l3 == 0);
  n[0] = p1_pieces(plain ? 3 : l1, (sep & 1) != 0, (sep & 2) != 0, pc[0]);
  n[1] = p1_pieces(plain ? 3 : l2, (sep & 4) != 0, (sep & 8) != 0, pc[1]);
  n[2] = p1_pieces(plain ? 3 : l3, (sep & 16) != 0, (sep & 32) != 0, pc[2]);
  clev = plain ? lev + 1 : lev;
}

// the split's count pass: the pieces of every flagged cloud (np) and its separation flags
__global__ void k_split_count(PCtx P, MCtx M, Ind d, SplitCtl C, int *np, int *sep) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const int code = P.i(DUSTB_PLEV, p);
  const double x[3] = {P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p), P.r(DUSTB_IPZ, p)};
  const int m = leaf_anchor(M, d, P.i(DUSTB_PGID, p));
  int n = 0, s = 0;
  if ((code & ~kCodeBits) == 0 && p1_flag(M, d, C, m, code, x)) {
    s = p1_sep(M, d, C, m, code, x);
    Piece pc[3][3]; int nn[3], clev;
    p1_build(code, s, pc, nn, clev);
    n = nn[0] * nn[1] * nn[2];
  }
  np[p] = (n > 0) ? n - 1 : 0;
  sep[p] = (n > 0) ? (s | 64) : 0;
}

// the split budget (:1062-1111): an event whose pieces start at or beyond the budget waits
// (its flags cleared, so the fill skips it); *taken receives the smallest such start, the
// pieces of the events taken (left as is when no event waits)
__global__ void k_split_budget(int *sep, const int *off, int n, long long budget, int *taken) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n || sep[p] == 0 || (long long)off[p] < budget) return;
  sep[p] = 0;
  atomicMin(taken, off[p]);
}

// WrapPos (:119-136) without shear: a piece into the domain; 1 if a physical x3 face mirrored it
__device__ __forceinline__ int leaf_wrap_pos(const MCtx &M, double c[3]) {
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  auto wrap = [](double x, double lo, double hi) {
    const double len = hi - lo;
    while (x < lo) x += len;
    while (x >= hi) x -= len;
    return x;
  };
  c[0] = wrap(c[0], M.x1min, M.x1max);
  c[1] = wrap(c[1], M.x2min, M.x2max);
  if (M.lt.x3per) { c[2] = wrap(c[2], M.x3min, M.x3max); return 0; }
  if (c[2] < M.x3min) { c[2] = 2.0 * M.x3min - c[2]; return 1; }
  if (c[2] >= M.x3max) {
    c[2] = 2.0 * M.x3max - c[2];
    if (c[2] >= M.x3max) c[2] = M.x3max - 1.0e-12 * L[2];
    return 1;
  }
  return 0;
}

// the split's fill (:1185-1243): the pieces, the parent's slot written last; off: the exclusive
// scan of the appended pieces
__global__ void k_split_fill(PCtx P, MCtx M, Ind d, const int *sep, const int *off,
                             unsigned long long tag0, int npart, int x3reflect) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npart || sep[p] == 0) return;
  const int code = P.i(DUSTB_PLEV, p);
  const double x[3] = {P.r(DUSTB_IPX, p), P.r(DUSTB_IPY, p), P.r(DUSTB_IPZ, p)};
  const double mass = P.r(DUSTB_IPM, p);
  Piece pc[3][3]; int n[3], clev;
  p1_build(code, sep[p] & 63, pc, n, clev);
  double e[3];
  for (int a = 0; a < 3; ++a) e[a] = half_width(M.lt, clev, a);
  const int n12 = n[0] * n[1];
  for (int k = n12 * n[2] - 1; k >= 0; --k) {
    const int ia[3] = {k % n[0], (k / n[0]) % n[1], k / n12};
    const int s = (k == 0) ? p : npart + off[p] + k - 1;
    double c[3];
    for (int a = 0; a < 3; ++a) c[a] = x[a] + pc[a][ia[a]].off * e[a];
    const int zmir = leaf_wrap_pos(M, c);
    if (k > 0) {
      for (int q = 0; q < DUSTB_NREAL; ++q) P.r(q, s) = P.r(q, p);
      for (int q = 0; q < DUSTB_NINT; ++q) P.i(q, s) = P.i(q, p);
      const unsigned long long t = tag0 + (unsigned long long)(off[p] + k - 1);
      P.i(DUSTB_PTAG, s) = (int)(unsigned)(t & 0xffffffffULL);
      P.i(DUSTB_PTAGH, s) = (int)(unsigned)(t >> 32);
    }
    P.r(DUSTB_IPX, s) = c[0]; P.r(DUSTB_IPX1, s) = c[0];
    P.r(DUSTB_IPY, s) = c[1]; P.r(DUSTB_IPY1, s) = c[1];
    P.r(DUSTB_IPZ, s) = c[2]; P.r(DUSTB_IPZ1, s) = c[2];
    const double mp = mass * pc[0][ia[0]].frac * pc[1][ia[1]].frac * pc[2][ia[2]].frac;
    const int l3 = pc[2][ia[2]].lobe;
    const int code_s = clev | (pc[0][ia[0]].lobe << kCodeLobe1) | (pc[1][ia[1]].lobe << kCodeLobe2) |
                       ((zmir ? ((l3 == 1 || l3 == 2) ? 3 - l3 : l3) : l3) << kCodeLobe3);
    P.r(DUSTB_IPM, s) = mp;
    P.i(DUSTB_PLEV, s) = code_s;
    if (zmir && x3reflect) { P.r(DUSTB_IPVZ, s) = -P.r(DUSTB_IPVZ, s); P.r(DUSTB_IPVZ1, s) = -P.r(DUSTB_IPVZ1, s); }
    const int am = leaf_anchor(M, d, P.i(DUSTB_PGID, s));
    const int b = leaf_owner(M, d, c, am);
    P.i(DUSTB_PGID, s) = M.gids + ((b >= 0 && b < d.nmb) ? b : am);
  }
}


// every leaf of the cloud at x (level lev, anchored at block m): f(leaf); with kMoments the
// moment traversal (a leaf with zero weight but a moment visited), else the weight traversal
template <bool kMoments, int LF, typename F>
__device__ void cloud_leaves(const MCtx &M, const Ind &d, int m, const double x[3], int lev,
                             const double L[3], int x3phys, F &&f, unsigned *err) {
  if constexpr (LF != 0) {
    leaf_foreach<kMoments>(M, d, m, x, lev, f);
    return;
  }
  CloudAxis X, Y, Z;
  cloud_axis(M, d, m, 0, x[0], lev, L[0], X);
  cloud_axis(M, d, m, 1, x[1], lev, L[1], Y);
  if (d.three_d) {
    cloud_axis(M, d, m, 2, x[2], lev, L[2], Z);
  } else {
    Z.n = 1; Z.o[0] = 0; Z.i[0] = 0; Z.w[0] = 1.0; Z.g[0] = 0.0; Z.org[0] = 0.0;
  }
  int npz = 1;
  double zp = x[2];
  if (x3phys && d.three_d) {
    const double ell = ldexp(M.s(m, DX3), -lev);
    const double lo = x[2] - ell, hi = x[2] + ell;
    if (lo < M.x3min || hi > M.x3max) {
      npz = 2;
      zp = 2.0 * ((hi > M.x3max) ? M.x3max : M.x3min) - x[2];
    }
  }
  for (int part = 0; part < npz; ++part) {
    if (part == 1) cloud_axis(M, d, m, 2, zp, lev, L[2], Z);
    for (int kz = 0; kz < Z.n; ++kz) {
      const double w3 = Z.w[kz], g3 = Z.g[kz];
      if (w3 == 0.0 && (!kMoments || g3 == 0.0)) continue;
      double czk = 0.0;
      if (kMoments && part == 1) {
        const double zc = Z.org[kz] + (Z.i[kz] + 0.5) * M.s(m, DX3);
        const double ez = x[2] - zc;
        czk = (zp - zc) - (ez - L[2] * round(ez / L[2]));
      }
      for (int jy = 0; jy < Y.n; ++jy) {
        const double w2 = Y.w[jy], g2 = Y.g[jy];
        if (w2 == 0.0 && (!kMoments || g2 == 0.0)) continue;
        const double w23 = w2 * w3;
        for (int ix = 0; ix < X.n; ++ix) {
          const double wa = X.w[ix];
          CloudLeaf lf;
          lf.w = w23 * wa;
          lf.m1x = lf.m1y = lf.m1z = 0.0;
          if (kMoments) {
            lf.m1x = w23 * X.g[ix];
            lf.m1y = wa * g2 * w3;
            lf.m1z = wa * w2 * g3;
            if (part == 1) lf.m1z += czk * lf.w;
            if (lf.w == 0.0 && lf.m1x == 0.0 && lf.m1y == 0.0 && lf.m1z == 0.0) continue;
          } else if (lf.w == 0.0) {
            continue;
          }
          lf.b = cloud_owner(M, d, m, X.o[ix], Y.o[jy], Z.o[kz]);
          if (lf.b < 0) { if (err) report(err, DUSTB_ERR_CLOUD); continue; }
          lf.k = d.ks + Z.i[kz]; lf.j = d.js + Y.i[jy]; lf.i = d.is + X.i[ix];
          f(lf);
        }
      }
    }
  }
}

// the clouds' linear gather of the packed field at x (CloudLinearGather3D without the blend)
template <int LF>
__device__ void cloud_gather(const MCtx &M, const Ind &d, int m, const double x[3], int lev,
                             const double L[3], int x3phys, const double *gp, double ug[3],
                             unsigned *err) {
  ug[0] = ug[1] = ug[2] = 0.0;
  cloud_leaves<true, LF>(M, d, m, x, lev, L, x3phys, [&](const CloudLeaf &lf) {
    const int b = lf.b;
    const double w = lf.w;
    const double dx1 = M.s(b, DX1), dx2 = M.s(b, DX2), dx3 = M.s(b, DX3);
    const double xc = M.s(b, X1MIN) + (lf.i - d.is + 0.5) * dx1;
    const double yc = M.s(b, X2MIN) + (lf.j - d.js + 0.5) * dx2;
    const double ex = x[0] - xc, ey = x[1] - yc;
    const double cx = 0.5 * (lf.m1x + (ex - L[0] * round(ex / L[0])) * w) / dx1;
    const double cy = 0.5 * (lf.m1y + (ey - L[1] * round(ey / L[1])) * w) / dx2;
    const double *g = gp + ((((long long)b * d.n3 + lf.k) * d.n2 + lf.j) * d.n1 + lf.i) * 12;
    if (d.three_d) {
      const double zc = M.s(b, X3MIN) + (lf.k - d.ks + 0.5) * dx3;
      const double ez = x[2] - zc;
      const double cz = 0.5 * (lf.m1z + (ez - L[2] * round(ez / L[2])) * w) / dx3;
      ug[0] += w * g[0] + cx * g[3] + cy * g[6] + cz * g[9];
      ug[1] += w * g[1] + cx * g[4] + cy * g[7] + cz * g[10];
      ug[2] += w * g[2] + cx * g[5] + cy * g[8] + cz * g[11];
    } else {
      ug[0] += w * g[0] + cx * g[3] + cy * g[6];
      ug[1] += w * g[1] + cx * g[4] + cy * g[7];
      ug[2] += w * g[2] + cx * g[5] + cy * g[8];
    }
  }, err);
}

// Every cloud kernel below is a body templated on the traversal form and two kernels: _u over
// the uniform-mesh traversal (no launch bounds: the compiler keeps it near 120 registers and 16
// warps per SM), _l over the leaf tables of refined meshes (held to 128 registers, 2 CTAs of 256
// threads per SM: about 15 % faster than its unbounded 230 registers, which allow one CTA).

// CloudDepositImplicitT (src/dust/dust_imex3d.cpp:61-99): Q = m c W / V, P = Q v
template <int LF>
__device__ __forceinline__ void k_cloud_deposit_body(PCtx P, MCtx M, Ind d, double *qdep, double a_dt, double sh,
                                int x3phys, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  int m, lev;
  double x[3];
  if (!cloud_load(P, M, d, p, sh, L, m, x, lev)) { report(err, DUSTB_ERR_CLOUD); return; }
  const double mass_c = d.three_d ? P.r(DUSTB_IPM, p) * a_dt / (P.r(DUSTB_IPTS, p) + a_dt)
                                  : P.r(DUSTB_IPM, p) * (a_dt / (P.r(DUSTB_IPTS, p) + a_dt));
  const double vx = P.r(DUSTB_IPVX, p), vy = P.r(DUSTB_IPVY, p), vz = P.r(DUSTB_IPVZ, p);
  cloud_leaves<false, LF>(M, d, m, x, lev, L, x3phys, [&](const CloudLeaf &lf) {
    const double dw = mass_c * lf.w / cloud_measure(M, d, lf.b);
    atomicAdd(&qdep[d.at(lf.b, 5, 0, lf.k, lf.j, lf.i)], dw);
    atomicAdd(&qdep[d.at(lf.b, 5, 1, lf.k, lf.j, lf.i)], dw * vx);
    atomicAdd(&qdep[d.at(lf.b, 5, 2, lf.k, lf.j, lf.i)], dw * vy);
    atomicAdd(&qdep[d.at(lf.b, 5, 3, lf.k, lf.j, lf.i)], dw * vz);
  }, err);
}
__global__ void k_cloud_deposit_u(PCtx P, MCtx M, Ind d, double *qdep, double a_dt, double sh,
                                int x3phys, unsigned *err) { k_cloud_deposit_body<0>(P, M, d, qdep, a_dt, sh, x3phys, err); }
__global__ void __launch_bounds__(kThreads, 2) k_cloud_deposit_l(PCtx P, MCtx M, Ind d, double *qdep, double a_dt, double sh,
                                int x3phys, unsigned *err) { k_cloud_deposit_body<1>(P, M, d, qdep, a_dt, sh, x3phys, err); }

// PackGatherField3D (src/dust/dust_cloud3d.cpp:1319-1340): the velocity and its central
// differences, gp(m, k, j, i, 0..11), over the padded interior (the outer layer zero); 2-D
// (PackGatherField, src/dust/dust_pm.cpp:81-102): the plane ks, no x3 differences
__global__ void k_gather_pack(Ind d, const double *v, double *gp) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = d.cells();
  if (idx >= per * d.nmb) return;
  const int m = (int)(idx / per);
  long long r = idx - (long long)m * per;
  const int i = (int)(r % d.n1); r /= d.n1;
  const int j = (int)(r % d.n2);
  const int k = (int)(r / d.n2);
  double *g = gp + idx * 12;
  const bool kin = d.three_d ? (k >= 1 && k < d.n3 - 1) : (k == d.ks);
  const bool in = i >= 1 && i < d.n1 - 1 && j >= 1 && j < d.n2 - 1 && kin;
  for (int q = 0; q < 3; ++q) {
    if (!in) { g[q] = g[3 + q] = g[6 + q] = g[9 + q] = 0.0; continue; }
    g[q] = v[d.at(m, 3, q, k, j, i)];
    g[3 + q] = v[d.at(m, 3, q, k, j, i + 1)] - v[d.at(m, 3, q, k, j, i - 1)];
    g[6 + q] = v[d.at(m, 3, q, k, j + 1, i)] - v[d.at(m, 3, q, k, j - 1, i)];
    g[9 + q] = d.three_d ? v[d.at(m, 3, q, k + 1, j, i)] - v[d.at(m, 3, q, k - 1, j, i)] : 0.0;
  }
}

// CloudGatherKickT without the blend (src/dust/dust_imex3d.cpp:114-175; the linear gather of
// dust_imex3d_gather.hpp and dust_leaf_api.hpp:196-219): ubar = sum w u* + cx du/dx + cy du/dy
// + cz du/dz, cx = (m1x + MinImage(x - xc) w) / (2 dx); dv = c (ubar - v), v += dv,
// R = dv / a_dt; with back-reaction -m w dv / V into dmom over the leaves of nonzero weight
template <int LF>
__device__ __forceinline__ void k_cloud_gather_kick_body(PCtx P, MCtx M, Ind d, const double *gp, double *dmom,
                                    double a_dt, double sh, int br, int x3phys, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  int m, lev;
  double x[3];
  if (!cloud_load(P, M, d, p, sh, L, m, x, lev)) { report(err, DUSTB_ERR_CLOUD); return; }
  double ug[3];
  cloud_gather<LF>(M, d, m, x, lev, L, x3phys, gp, ug, err);
  const double cj = a_dt / (P.r(DUSTB_IPTS, p) + a_dt);
  const double dvx = cj * (ug[0] - P.r(DUSTB_IPVX, p));
  const double dvy = cj * (ug[1] - P.r(DUSTB_IPVY, p));
  const double dvz = cj * (ug[2] - P.r(DUSTB_IPVZ, p));
  P.r(DUSTB_IPVX, p) += dvx; P.r(DUSTB_IPVY, p) += dvy; P.r(DUSTB_IPVZ, p) += dvz;
  P.r(DUSTB_IPRX, p) = dvx / a_dt; P.r(DUSTB_IPRY, p) = dvy / a_dt; P.r(DUSTB_IPRZ, p) = dvz / a_dt;
  if (!br) return;
  const double mass = -P.r(DUSTB_IPM, p);
  cloud_leaves<false, LF>(M, d, m, x, lev, L, x3phys, [&](const CloudLeaf &lf) {
    const double dw = mass * lf.w / cloud_measure(M, d, lf.b);
    atomicAdd(&dmom[d.at(lf.b, 3, 0, lf.k, lf.j, lf.i)], dw * dvx);
    atomicAdd(&dmom[d.at(lf.b, 3, 1, lf.k, lf.j, lf.i)], dw * dvy);
    atomicAdd(&dmom[d.at(lf.b, 3, 2, lf.k, lf.j, lf.i)], dw * dvz);
  }, nullptr);
}
__global__ void k_cloud_gather_kick_u(PCtx P, MCtx M, Ind d, const double *gp, double *dmom,
                                    double a_dt, double sh, int br, int x3phys, unsigned *err) { k_cloud_gather_kick_body<0>(P, M, d, gp, dmom, a_dt, sh, br, x3phys, err); }
__global__ void __launch_bounds__(kThreads, 2) k_cloud_gather_kick_l(PCtx P, MCtx M, Ind d, const double *gp, double *dmom,
                                    double a_dt, double sh, int br, int x3phys, unsigned *err) { k_cloud_gather_kick_body<1>(P, M, d, gp, dmom, a_dt, sh, br, x3phys, err); }

// CloudOperatorKernelT (src/dust/dust_cloud_imex_kernels.hpp:20-70): the clouds' m c W ubar / V
// with ubar their linear gather of the packed field, into result (the operator of dc1 / dc2)
template <int LF>
__device__ __forceinline__ void k_cloud_operator_body(PCtx P, MCtx M, Ind d, const double *gp, double *result,
                                 double a_dt, double sh, int x3phys, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  int m, lev;
  double x[3];
  if (!cloud_load(P, M, d, p, sh, L, m, x, lev)) { report(err, DUSTB_ERR_CLOUD); return; }
  double ug[3];
  cloud_gather<LF>(M, d, m, x, lev, L, x3phys, gp, ug, err);
  const double mc = P.r(DUSTB_IPM, p) * (a_dt / (P.r(DUSTB_IPTS, p) + a_dt));
  cloud_leaves<false, LF>(M, d, m, x, lev, L, x3phys, [&](const CloudLeaf &lf) {
    const double dw = mc * lf.w / cloud_measure(M, d, lf.b);
    atomicAdd(&result[d.at(lf.b, 3, 0, lf.k, lf.j, lf.i)], dw * ug[0]);
    atomicAdd(&result[d.at(lf.b, 3, 1, lf.k, lf.j, lf.i)], dw * ug[1]);
    atomicAdd(&result[d.at(lf.b, 3, 2, lf.k, lf.j, lf.i)], dw * ug[2]);
  }, nullptr);
}
__global__ void k_cloud_operator_u(PCtx P, MCtx M, Ind d, const double *gp, double *result,
                                 double a_dt, double sh, int x3phys, unsigned *err) { k_cloud_operator_body<0>(P, M, d, gp, result, a_dt, sh, x3phys, err); }
__global__ void __launch_bounds__(kThreads, 2) k_cloud_operator_l(PCtx P, MCtx M, Ind d, const double *gp, double *result,
                                 double a_dt, double sh, int x3phys, unsigned *err) { k_cloud_operator_body<1>(P, M, d, gp, result, a_dt, sh, x3phys, err); }

// CloudImplicitConsistencyOverlapT (src/dust/dust_imex3d.cpp:669-790), the cells: g = rho u* -
// M, r = (D - g) / (rho + Q) (by the reciprocal), the gas takes g + rho r, dmom its rate, r
// into res (vars 0-2 of a 4-variable field)
__global__ void k_cloud_consistent_gas(Ind d, double *u0, int nv, const double *us,
                                       const double *qdep, double *dmom, double *res,
                                       double inv_adt) {
  int m, k, j, i;
  if (!active_cell(d, blockIdx.x * (long long)blockDim.x + threadIdx.x, m, k, j, i)) return;
  const double rho = u0[d.at(m, nv, 0, k, j, i)];
  const double q = qdep[d.at(m, 5, 0, k, j, i)];
  const double inv = 1.0 / (rho + q);
  for (int v = 0; v < 3; ++v) {
    const long long a3 = d.at(m, 3, v, k, j, i), au = d.at(m, nv, 1 + v, k, j, i);
    const double g = rho * us[a3] - u0[au];
    const double r = (dmom[a3] - g) * inv;
    const double dgas = g + rho * r;
    u0[au] += dgas;
    dmom[a3] = dgas * inv_adt;
    res[d.at(m, 4, v, k, j, i)] = r;
  }
}

// ... the clouds: v += c sum W r, R += c sum W r / a_dt with the deposit's weights
template <int LF>
__device__ __forceinline__ void k_cloud_consistent_dust_body(PCtx P, MCtx M, Ind d, const double *res, double a_dt,
                                        double sh, int x3phys) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  if (P.r(DUSTB_IPM, p) <= 0.0) return;
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  int m, lev;
  double x[3];
  if (!cloud_load(P, M, d, p, sh, L, m, x, lev)) return;
  double rv[3] = {0.0, 0.0, 0.0};
  cloud_leaves<false, LF>(M, d, m, x, lev, L, x3phys, [&](const CloudLeaf &lf) {
    for (int v = 0; v < 3; ++v) rv[v] += lf.w * res[d.at(lf.b, 4, v, lf.k, lf.j, lf.i)];
  }, nullptr);
  const double cj = a_dt / (P.r(DUSTB_IPTS, p) + a_dt);
  P.r(DUSTB_IPVX, p) += cj * rv[0]; P.r(DUSTB_IPVY, p) += cj * rv[1]; P.r(DUSTB_IPVZ, p) += cj * rv[2];
  P.r(DUSTB_IPRX, p) += cj * rv[0] / a_dt;
  P.r(DUSTB_IPRY, p) += cj * rv[1] / a_dt;
  P.r(DUSTB_IPRZ, p) += cj * rv[2] / a_dt;
}
__global__ void k_cloud_consistent_dust_u(PCtx P, MCtx M, Ind d, const double *res, double a_dt,
                                        double sh, int x3phys) { k_cloud_consistent_dust_body<0>(P, M, d, res, a_dt, sh, x3phys); }
__global__ void __launch_bounds__(kThreads, 2) k_cloud_consistent_dust_l(PCtx P, MCtx M, Ind d, const double *res, double a_dt,
                                        double sh, int x3phys) { k_cloud_consistent_dust_body<1>(P, M, d, res, a_dt, sh, x3phys); }

// ---- the clouds' pc2 (src/dust/dust_cloud3d.cpp:1362-1538, CloudPC2Push :76-150) ----------
// PackGasGather3D: the gas velocity u1 momentum / density in every cell
__global__ void k_gas_velocity_all(Ind d, const double *u, int nv, double *uv) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = d.cells();
  if (idx >= per * d.nmb) return;
  const int m = (int)(idx / per);
  const long long r = idx - (long long)m * per;
  const long long base = (long long)m * nv * per;
  const double invrho = 1.0 / u[base + r];
  for (int v = 0; v < 3; ++v) uv[((long long)m * 3 + v) * per + r] = u[base + (1 + v) * per + r] * invrho;
}

// CloudPredictorT: g = -dt (m / t_s) (ubar - v) into qdep 1-3, m / t_s into qdep 4 (rate_dep)
template <int LF>
__device__ __forceinline__ void k_cloud_pc2_predictor_body(PCtx P, MCtx M, Ind d, const double *gp, double *qdep,
                                      double dt, int rate_dep, int x3phys, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  int m, lev;
  double x[3];
  if (!cloud_load(P, M, d, p, 0.0, L, m, x, lev)) { report(err, DUSTB_ERR_CLOUD); return; }
  double ug[3];
  cloud_gather<LF>(M, d, m, x, lev, L, x3phys, gp, ug, err);
  const double mass_rate = P.r(DUSTB_IPM, p) / P.r(DUSTB_IPTS, p);
  const double gx = -dt * mass_rate * (ug[0] - P.r(DUSTB_IPVX, p));
  const double gy = -dt * mass_rate * (ug[1] - P.r(DUSTB_IPVY, p));
  const double gz = -dt * mass_rate * (ug[2] - P.r(DUSTB_IPVZ, p));
  cloud_leaves<false, LF>(M, d, m, x, lev, L, x3phys, [&](const CloudLeaf &lf) {
    const double inv_volume = 1.0 / cloud_measure(M, d, lf.b);
    atomicAdd(&qdep[d.at(lf.b, 5, 1, lf.k, lf.j, lf.i)], inv_volume * lf.w * gx);
    atomicAdd(&qdep[d.at(lf.b, 5, 2, lf.k, lf.j, lf.i)], inv_volume * lf.w * gy);
    atomicAdd(&qdep[d.at(lf.b, 5, 3, lf.k, lf.j, lf.i)], inv_volume * lf.w * gz);
    if (rate_dep) atomicAdd(&qdep[d.at(lf.b, 5, 4, lf.k, lf.j, lf.i)], inv_volume * lf.w * mass_rate);
  }, nullptr);
}
__global__ void k_cloud_pc2_predictor_u(PCtx P, MCtx M, Ind d, const double *gp, double *qdep,
                                      double dt, int rate_dep, int x3phys, unsigned *err) { k_cloud_pc2_predictor_body<0>(P, M, d, gp, qdep, dt, rate_dep, x3phys, err); }
__global__ void __launch_bounds__(kThreads, 2) k_cloud_pc2_predictor_l(PCtx P, MCtx M, Ind d, const double *gp, double *qdep,
                                      double dt, int rate_dep, int x3phys, unsigned *err) { k_cloud_pc2_predictor_body<1>(P, M, d, gp, qdep, dt, rate_dep, x3phys, err); }

// CloudAdvanceT with CloudPC2Push's Midpoint / Kick / Drift
template <int LF>
__device__ __forceinline__ void k_cloud_pc2_advance_body(PCtx P, MCtx M, Ind d, const double *gp, double *dmom,
                                    double dt, int br, int sbox, int strat, double q, double om,
                                    double aphi, int x3phys, unsigned *err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P.npart) return;
  const double L[3] = {M.x1max - M.x1min, M.x2max - M.x2min, M.x3max - M.x3min};
  const int m = P.i(DUSTB_PGID, p) - M.gids, lev = P.i(DUSTB_PLEV, p);
  const double x0[3] = {P.r(DUSTB_IPX1, p), P.r(DUSTB_IPY1, p), d.three_d ? P.r(DUSTB_IPZ1, p) : 0.0};
  const double v0[3] = {P.r(DUSTB_IPVX1, p), P.r(DUSTB_IPVY1, p), P.r(DUSTB_IPVZ1, p)};
  double xh[3], xg[3];
  if (d.three_d) {
    xh[0] = x0[0] + 0.5 * dt * v0[0];
    xh[1] = x0[1] + 0.5 * dt * (v0[1] - (sbox ? q * om * x0[0] : 0.0));
    xh[2] = x0[2] + 0.5 * dt * v0[2];
    xg[0] = xh[0];
    xg[1] = xh[1] + (sbox ? q * om * xh[0] * 0.5 * dt : 0.0);
    xg[2] = xh[2];
  } else {
    xh[0] = x0[0] + 0.5 * dt * v0[0];
    xh[1] = x0[1] + 0.5 * dt * v0[1];
    xh[2] = x0[2];
    xg[0] = xh[0]; xg[1] = xh[1]; xg[2] = xh[2];
  }
  double x[3] = {xg[0], xg[1], xg[2]};
  if (!cloud_frame_ok(M, d, m, lev, L, x, 1.0)) { report(err, DUSTB_ERR_CLOUD); return; }
  double ug[3];
  cloud_gather<LF>(M, d, m, x, lev, L, x3phys, gp, ug, err);
  const double h = 0.5 * dt;
  const double lambda = h / P.r(DUSTB_IPTS, p);
  const double aa = 1.0 + lambda;
  double r[3] = {v0[0] + lambda * ug[0], v0[1] + lambda * ug[1], v0[2] + lambda * ug[2]};
  double vh[3];
  if (d.three_d) {
    if (sbox) {
      const double cxy = 2.0 * h * om, cyx = h * (2.0 - q) * om;
      const double det = aa * aa + cxy * cyx;
      vh[0] = (aa * r[0] + cxy * r[1]) / det;
      vh[1] = (aa * r[1] - cyx * r[0]) / det;
      if (strat) r[2] -= h * (om * om) * xh[2];
      vh[2] = r[2] / aa;
    } else {
      vh[0] = r[0] / aa; vh[1] = r[1] / aa; vh[2] = r[2] / aa;
    }
  } else {
    if (sbox) {
      const double cxz = 2.0 * h * om, czx = h * (2.0 - q) * om;
      const double det = aa * aa + cxz * czx;
      if (aphi != 0.0) r[2] += h * aphi;
      vh[0] = (aa * r[0] + cxz * r[2]) / det;
      vh[2] = (aa * r[2] - czx * r[0]) / det;
      vh[1] = r[1] / aa;
    } else {
      vh[0] = r[0] / aa; vh[1] = r[1] / aa; vh[2] = r[2] / aa;
    }
  }
  P.r(DUSTB_IPVX, p) = 2.0 * vh[0] - v0[0];
  P.r(DUSTB_IPVY, p) = 2.0 * vh[1] - v0[1];
  P.r(DUSTB_IPVZ, p) = 2.0 * vh[2] - v0[2];
  P.r(DUSTB_IPX, p) = x0[0] + dt * vh[0];
  if (d.three_d) {
    P.r(DUSTB_IPY, p) = x0[1] + dt * (vh[1] - (sbox ? q * om * xh[0] : 0.0));
    P.r(DUSTB_IPZ, p) = x0[2] + dt * vh[2];
  } else {
    P.r(DUSTB_IPY, p) = x0[1] + dt * vh[1];
  }
  P.r(DUSTB_IPX1, p) = xh[0]; P.r(DUSTB_IPY1, p) = xh[1];
  if (d.three_d) P.r(DUSTB_IPZ1, p) = xh[2];
  const double dvx = dt * (ug[0] - vh[0]) / P.r(DUSTB_IPTS, p);
  const double dvy = dt * (ug[1] - vh[1]) / P.r(DUSTB_IPTS, p);
  const double dvz = dt * (ug[2] - vh[2]) / P.r(DUSTB_IPTS, p);
  P.r(DUSTB_IPRX, p) = dvx; P.r(DUSTB_IPRY, p) = dvy; P.r(DUSTB_IPRZ, p) = dvz;
  if (!br) return;
  const double mass = -P.r(DUSTB_IPM, p);
  cloud_leaves<false, LF>(M, d, m, x, lev, L, x3phys, [&](const CloudLeaf &lf) {
    const double dw = mass * lf.w / cloud_measure(M, d, lf.b);
    atomicAdd(&dmom[d.at(lf.b, 3, 0, lf.k, lf.j, lf.i)], dw * dvx);
    atomicAdd(&dmom[d.at(lf.b, 3, 1, lf.k, lf.j, lf.i)], dw * dvy);
    atomicAdd(&dmom[d.at(lf.b, 3, 2, lf.k, lf.j, lf.i)], dw * dvz);
  }, nullptr);
}
__global__ void k_cloud_pc2_advance_u(PCtx P, MCtx M, Ind d, const double *gp, double *dmom,
                                    double dt, int br, int sbox, int strat, double q, double om,
                                    double aphi, int x3phys, unsigned *err) { k_cloud_pc2_advance_body<0>(P, M, d, gp, dmom, dt, br, sbox, strat, q, om, aphi, x3phys, err); }
__global__ void __launch_bounds__(kThreads, 2) k_cloud_pc2_advance_l(PCtx P, MCtx M, Ind d, const double *gp, double *dmom,
                                    double dt, int br, int sbox, int strat, double q, double om,
                                    double aphi, int x3phys, unsigned *err) { k_cloud_pc2_advance_body<1>(P, M, d, gp, dmom, dt, br, sbox, strat, q, om, aphi, x3phys, err); }

long long n_active(const Ind &d) { return (long long)d.nmb * d.nx3 * d.nx2 * d.nx1; }
long long n_all(const Ind &d) { return d.cells() * d.nmb; }

bool ctx_ok(const dustb_ctx *c) {
  if (!c) return false;
  const dustb_mesh &m = c->mesh;
  if (m.nmb <= 0 || m.nx1 <= 0 || m.ng < 2 || !m.mb_size || !m.nghbr || !m.multi_d) return false;
  if (m.three_d && m.nx3 <= 0) return false;
  // every ghost cell must map to an active cell of one neighbour
  if (m.nx1 < m.ng || (m.multi_d && m.nx2 < m.ng) || (m.three_d && m.nx3 < m.ng)) return false;
  if (c->part.npart < 0 || (c->part.npart > 0 && (!c->part.pr || !c->part.pi))) return false;
  if (c->part.npart > c->part.stride) return false;
  if (c->f.nvar_gas < 4) return false;
  return true;
}

// the context of a task that reads no particle row (the per-cell solves and exchanges, the
// mixed form's cycles): the particle rows may be detached (pr = pi = NULL, npart kept)
bool ctx_cells_ok(const dustb_ctx *c) {
  if (!c) return false;
  if (!c->part.pr && !c->part.pi && c->part.npart >= 0) {
    dustb_ctx d = *c;
    d.part.npart = 0;
    return ctx_ok(&d);
  }
  return ctx_ok(c);
}

}  // namespace

// ---- host error bookkeeping --------------------------------------------------------------
namespace dustb_host {
static char g_err[256] = "";
void set_error(const char *what, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
}
void set_message(const char *what) { snprintf(g_err, sizeof(g_err), "%s", what); }
int launch_status(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_error(what, e); return DUSTB_ELAUNCH; }
  return DUSTB_OK;
}
}  // namespace dustb_host

using dustb_host::launch_status;

// launchers of the per-cell FP64 kernels, shared with the mixed-precision form
namespace dustb_cells {
void gas_rk(const dustb_ctx *c, double g0, double g1, cudaStream_t st) {
  Ind d = make_ind(c->mesh);
  k_gas_rk<<<blocks_for(n_active(d)), kThreads, 0, st>>>(d, c->f.u0, c->f.u1, c->f.nvar_gas, g0, g1);
}
void history(const dustb_ctx *c, double atw_dt, cudaStream_t st) {
  Ind d = make_ind(c->mesh);
  k_history<<<blocks_for(n_active(d)), kThreads, 0, st>>>(d, c->f.u0, c->f.nvar_gas, c->f.dmom,
                                                          nullptr, atw_dt);
}
// u0.m += atw_dt dmom, then u0.m += atw_dt f for a 3-variable field f (the mixed form's rate
// ledger), in one pass: the same sums as two history launches
void history_field(const dustb_ctx *c, const double *f, double atw_dt, cudaStream_t st) {
  Ind d = make_ind(c->mesh);
  k_history<<<blocks_for(n_active(d)), kThreads, 0, st>>>(d, c->f.u0, c->f.nvar_gas, c->f.dmom, f,
                                                          atw_dt);
}
void dc_correct(const dustb_ctx *c, cudaStream_t st) {
  Ind d = make_ind(c->mesh);
  k_dc_correct<<<blocks_for(n_active(d)), kThreads, 0, st>>>(d, c->f.u0, c->f.nvar_gas, c->f.qdep,
                                                             c->f.work, c->f.ustar);
}
void consistent_gas(const dustb_ctx *c, double a_dt, cudaStream_t st) {
  Ind d = make_ind(c->mesh);
  k_consistent_gas<<<blocks_for(n_active(d)), kThreads, 0, st>>>(
      d, c->f.u0, c->f.nvar_gas, c->f.ustar, c->f.qdep, c->f.dmom, c->f.resid, 1.0 / a_dt);
}
void pmbr(const dustb_ctx *c, double a_dt, cudaStream_t st) {
  Ind d = make_ind(c->mesh);
  k_pmbr<<<blocks_for(n_active(d)), kThreads, 0, st>>>(d, c->f.u0, c->f.nvar_gas, c->f.dmom, 1.0 / a_dt);
}
bool ctx_valid(const dustb_ctx *c) { return ctx_cells_ok(c); }
}  // namespace dustb_cells

#define CHECK_CTX(c) do { if (!ctx_ok(c)) { return DUSTB_EINVAL; } } while (0)
#define CHECK_CELLS(c) do { if (!ctx_cells_ok(c)) { return DUSTB_EINVAL; } } while (0)
#define PGRID(c) blocks_for((c)->part.npart), kThreads, 0, S(stream)

extern "C" {

int dustb_version(void) { return 1; }
const char *dustb_last_error(void) { return dustb_host::g_err; }

int dustb_register_copy(const dustb_ctx *c, void *stream) {
  CHECK_CTX(c);
  Ind d = make_ind(c->mesh);
  size_t bytes = (size_t)n_all(d) * c->f.nvar_gas * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(c->f.u1, c->f.u0, bytes, cudaMemcpyDeviceToDevice, S(stream));
  if (e != cudaSuccess) { dustb_host::set_error("register_copy", e); return DUSTB_ELAUNCH; }
  if (c->part.npart > 0) k_reg_copy<<<PGRID(c)>>>(pview(c));
  return launch_status("register_copy");
}

int dustb_gas_rk_noflux(const dustb_ctx *c, double gam0, double gam1, void *stream) {
  CHECK_CELLS(c);
  Ind d = make_ind(c->mesh);
  k_gas_rk<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.u1, c->f.nvar_gas, gam0, gam1);
  return launch_status("gas_rk_noflux");
}

int dustb_history_gas(const dustb_ctx *c, double atw_dt, void *stream) {
  CHECK_CELLS(c);
  Ind d = make_ind(c->mesh);
  k_history<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas, c->f.dmom, nullptr, atw_dt);
  return launch_status("history_gas");
}

int dustb_push_imex(const dustb_ctx *c, double gam0, double gam1, double beta_dt, double atw_dt,
                    void *stream) {
  CHECK_CTX(c);
  if (c->part.npart == 0) return DUSTB_OK;
  k_push_imex<<<PGRID(c)>>>(pview(c), c->mesh.three_d, c->phys.shearing_box, c->phys.stratified,
                            c->phys.qshear, c->phys.omega0, gam0, gam1, beta_dt, atw_dt);
  return launch_status("push_imex");
}

int dustb_route(const dustb_ctx *c, double *x3_removed, void *stream) {
  CHECK_CTX(c);
  if (c->mesh.x3bc == DUSTB_X3_OUTFLOW && !x3_removed) return DUSTB_EINVAL;
  if (c->part.npart == 0) return DUSTB_OK;
  Ind d = make_ind(c->mesh);
  const SBox B = sbview(c);
  if (B.on && (!B.sb_gid || B.nb2 <= 0 || B.nb3 <= 0)) return DUSTB_EINVAL;
  // refined meshes: 3-D, both tables, no shear-periodic faces (their maps are single-level)
  if ((c->mesh.nghbr_ml != nullptr) != (c->mesh.mb_lev != nullptr)) return DUSTB_EINVAL;
  if (c->mesh.nghbr_ml && (!c->mesh.three_d || B.on)) return DUSTB_EUNSUP;
  k_route<<<PGRID(c)>>>(pview(c), mview(c), d, c->mesh.x3bc, x3_removed, c->err, B);
  return launch_status("route");
}

int dustb_deposit_qp(const dustb_ctx *c, double a_dt, double sh, void *stream) {
  CHECK_CTX(c);
  Ind d = make_ind(c->mesh);
  cudaMemsetAsync(c->f.qdep, 0, (size_t)n_all(d) * 5 * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_scatter<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.qdep, a_dt, sh, c->err);
  return launch_status("deposit_qp");
}

int dustb_ghost_add(const dustb_ctx *c, double *field, int nvar, void *stream) {
  CHECK_CELLS(c);
  if (!field || nvar <= 0) return DUSTB_EINVAL;
  if (c->mesh.nghbr_ml) return DUSTB_EUNSUP;        // refined: dustb_ghost_add_plan
  Ind d = make_ind(c->mesh);
  const int fold = d.three_d && c->mesh.x3bc != DUSTB_X3_PERIODIC && !c->phys.x3_deposit_drop;
  const SBox B = sbview(c);
  k_ghost_add<<<blocks_for(make_shell(d).per * d.nmb * nvar), kThreads, 0, S(stream)>>>(d, c->mesh.nghbr, c->mesh.gids, field, nvar, fold,
                                                                          B);
  if (B.on) {
    if (!B.sb_gid || B.nb2 <= 0 || B.nb3 <= 0) return DUSTB_EINVAL;
    k_shear_add<<<blocks_for((long long)d.nmb * nvar * d.nx3 * d.nx2 * 2 * d.ng), kThreads, 0, S(stream)>>>(
        d, B, field, nvar);
  }
  return launch_status("ghost_add");
}

int dustb_ghost_add_plan(const dustb_ctx *c, const dustb_dep_plan *plan, double *field,
                         int nvar, void *stream) {
  CHECK_CELLS(c);
  if (!plan || !field || nvar <= 0 || plan->nseg < 0 || !c->mesh.three_d) return DUSTB_EINVAL;
  if (plan->nseg == 0) return DUSTB_OK;
  if (!plan->seg_tgt || !plan->seg_ptr || !plan->ent_src || !plan->ent_w) return DUSTB_EINVAL;
  Ind d = make_ind(c->mesh);
  k_dep_plan_apply<<<blocks_for((long long)plan->nseg * nvar), kThreads, 0, S(stream)>>>(
      plan->nseg, plan->seg_tgt, plan->seg_ptr, plan->ent_src, plan->ent_w, field, nvar,
      d.cells());
  return launch_status("ghost_add_plan");
}

int dustb_ghost_copy(const dustb_ctx *c, double *field, int nvar, int x3_bcs, void *stream) {
  CHECK_CELLS(c);
  if (!field || nvar <= 0) return DUSTB_EINVAL;
  if (c->mesh.nghbr_ml) return DUSTB_EUNSUP;        // (no prolongation across levels)
  Ind d = make_ind(c->mesh);
  k_ghost_copy<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(d, c->mesh.nghbr, c->mesh.gids, field, nvar);
  const SBox B = sbview(c);
  if (B.on) {
    // the shearing box remap of the x1 ghost strips, after the plain copy and before the
    // x3 boundary values (RecvUstar -> RecvUstarShr -> FinishUstarGhosts, dust_tasks.cpp)
    if (!B.sb_gid || B.nb2 <= 0 || B.nb3 <= 0) return DUSTB_EINVAL;
    k_shear_copy<<<blocks_for(2LL * B.nb3 * B.nb2 * nvar * d.n3 * d.n2 * d.ng), kThreads, 0, S(stream)>>>(
        B, d, field, nvar);
  }
  if (x3_bcs && nvar == 3 && d.three_d && c->mesh.x3bc != DUSTB_X3_PERIODIC)
    k_x3_bcs<<<blocks_for((long long)d.ng * d.n2 * d.n1 * d.nmb), kThreads, 0, S(stream)>>>(
        d, c->mesh.nghbr, field, c->mesh.x3bc == DUSTB_X3_REFLECT);
  return launch_status("ghost_copy");
}

int dustb_solve_ustar(const dustb_ctx *c, void *stream) {
  CHECK_CELLS(c);
  Ind d = make_ind(c->mesh);
  k_solve_ustar<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas, c->f.qdep,
                                                                     c->f.ustar, c->phys.back_reaction);
  return launch_status("solve_ustar");
}

int dustb_dc1_sweep(const dustb_ctx *c, double a_dt, double sh, void *stream) {
  CHECK_CTX(c);
  Ind d = make_ind(c->mesh);
  int rc = dustb_ghost_copy(c, c->f.ustar, 3, 1, stream);
  if (rc) return rc;
  cudaMemsetAsync(c->f.work, 0, (size_t)n_all(d) * 3 * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_operator<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.ustar, c->f.work, a_dt, sh, c->err);
  rc = dustb_ghost_add(c, c->f.work, 3, stream);
  if (rc) return rc;
  k_dc_correct<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas, c->f.qdep,
                                                                    c->f.work, c->f.ustar);
  return launch_status("dc1_sweep");
}

int dustb_gather_kick_pmbr(const dustb_ctx *c, double a_dt, double sh, void *stream) {
  CHECK_CTX(c);
  Ind d = make_ind(c->mesh);
  const int br = c->phys.back_reaction;
  if (br) cudaMemsetAsync(c->f.dmom, 0, (size_t)n_all(d) * 3 * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_gather_kick<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.ustar, c->f.dmom, a_dt, sh, br, c->err);
  return launch_status("gather_kick_pmbr");
}

int dustb_apply_pmbr(const dustb_ctx *c, double a_dt, void *stream) {
  CHECK_CTX(c);
  if (!c->phys.back_reaction) return DUSTB_OK;
  Ind d = make_ind(c->mesh);
  const double inv_adt = 1.0 / a_dt;
  if (!c->phys.consistent_gas) {
    k_pmbr<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas, c->f.dmom, inv_adt);
    return launch_status("apply_pmbr");
  }
  cudaMemsetAsync(c->f.resid, 0, (size_t)n_all(d) * 4 * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_center_mass<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.resid, a_dt, c->err);
  k_consistent_gas<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(
      d, c->f.u0, c->f.nvar_gas, c->f.ustar, c->f.qdep, c->f.dmom, c->f.resid, inv_adt);
  if (c->part.npart > 0)
    k_consistent_dust<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.resid, a_dt);
  return launch_status("apply_pmbr");
}

int dustb_newdt(const dustb_ctx *c, double dt_cfl, double *dt_out, void *stream) {
  CHECK_CTX(c);
  if (!dt_out) return DUSTB_EINVAL;
  Ind d = make_ind(c->mesh);
  k_set<<<1, 1, 0, S(stream)>>>(dt_out, (double)FLT_MAX, 0, 0.0);
  if (c->part.npart > 0)
    k_newdt<<<PGRID(c)>>>(pview(c), mview(c), d, c->phys.shearing_box && d.three_d,
                          c->phys.qshear * c->phys.omega0, dt_out);
  k_scale<<<1, 1, 0, S(stream)>>>(dt_out, dt_cfl);
  return launch_status("newdt");
}

int dustb_tstop_extrema(const dustb_ctx *c, double *out, void *stream) {
  CHECK_CTX(c);
  if (!out) return DUSTB_EINVAL;
  k_set<<<1, 1, 0, S(stream)>>>(out, 0.0, 1, DBL_MAX);
  if (c->part.npart > 0) k_tstop<<<PGRID(c)>>>(pview(c), out, c->err);
  return launch_status("tstop_extrema");
}

int dustb_pc2_predictor(const dustb_ctx *c, double dt, int rate_dep, void *stream) {
  CHECK_CTX(c);
  Ind d = make_ind(c->mesh);
  cudaMemsetAsync(c->f.qdep, 0, (size_t)n_all(d) * 5 * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_pc2_predictor<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.u1, c->f.nvar_gas, c->f.qdep, dt,
                                  rate_dep, c->err);
  return launch_status("pc2_predictor");
}

int dustb_pc2_apply_predictor(const dustb_ctx *c, double dt, double *chi_max, void *stream) {
  CHECK_CELLS(c);
  Ind d = make_ind(c->mesh);
  if (chi_max) {
    k_set<<<1, 1, 0, S(stream)>>>(chi_max, 0.0, 0, 0.0);
    k_pc2_rate_max<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas, c->f.qdep, chi_max);
    k_scale<<<1, 1, 0, S(stream)>>>(chi_max, dt);
  }
  k_pc2_apply<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas, c->f.qdep, dt,
                                                                   c->phys.pc2_feedback_damping);
  return launch_status("pc2_apply_predictor");
}

int dustb_pc2_midpoint(const dustb_ctx *c, void *stream) {
  CHECK_CELLS(c);
  Ind d = make_ind(c->mesh);
  k_pc2_midpoint<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.u1, c->f.nvar_gas, c->f.ustar);
  return launch_status("pc2_midpoint");
}

int dustb_pc2_advance(const dustb_ctx *c, double dt, void *stream) {
  CHECK_CTX(c);
  Ind d = make_ind(c->mesh);
  const int br = c->phys.back_reaction;
  if (br) cudaMemsetAsync(c->f.dmom, 0, (size_t)n_all(d) * 3 * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_pc2_advance<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.ustar, c->f.dmom, dt, br,
                                c->phys.shearing_box, c->phys.stratified, c->phys.qshear,
                                c->phys.omega0, c->phys.const_accel_phi, c->err);
  return launch_status("pc2_advance");
}

int dustb_pc2_commit(const dustb_ctx *c, double wpred, void *stream) {
  CHECK_CELLS(c);
  Ind d = make_ind(c->mesh);
  k_pc2_commit<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas, c->f.dmom,
                                                                    c->f.qdep, wpred);
  return launch_status("pc2_commit");
}

long long dustb_phst_scratch_bytes(const dustb_mesh *mesh, int npart) {
  if (!mesh) return -1;
  const Ind d = make_ind(*mesh);
  const long long nchunk = ((long long)(npart > 0 ? npart : 1) + kPhstChunk - 1) / kPhstChunk;
  const long long fb = d.cells() * d.nmb * 8;
  return ((nchunk * kPhstSums * 8 + 255) & ~255LL) + ((fb + 255) & ~255LL) + 1024 * 16;
}

int dustb_phst(const dustb_ctx *c, const double *chi_max, double *row, void *scratch,
               long long bytes, void *stream) {
  CHECK_CTX(c);
  if (!row) return DUSTB_EINVAL;
  if (!c->mesh.three_d) return DUSTB_EUNSUP;      // (the densest cell of point particles: 3-D)
  if (!scratch || bytes < dustb_phst_scratch_bytes(&c->mesh, c->part.npart)) return DUSTB_ESCRATCH;
  const Ind d = make_ind(c->mesh);
  const int np = c->part.npart;
  const int nchunk = (int)(((long long)(np > 0 ? np : 1) + kPhstChunk - 1) / kPhstChunk);
  char *b = (char *)scratch;
  double *part = (double *)b;
  b += ((long long)nchunk * kPhstSums * 8 + 255) & ~255LL;
  double *field = (double *)b;
  b += (d.cells() * d.nmb * 8 + 255) & ~255LL;
  double *bval = (double *)b;
  long long *bloc = (long long *)(b + 1024 * 8);
  cudaMemsetAsync(part, 0, (size_t)nchunk * kPhstSums * 8, S(stream));
  if (np > 0) k_phst_chunks<<<blocks_for(nchunk), kThreads, 0, S(stream)>>>(pview(c), DUSTB_IPZ, part, nchunk);
  k_phst_sums<<<1, 1, 0, S(stream)>>>(part, nchunk, chi_max, c->phys.back_reaction, row);
  cudaMemsetAsync(field, 0, (size_t)d.cells() * d.nmb * 8, S(stream));
  if (np > 0) k_mass_deposit<<<PGRID(c)>>>(pview(c), mview(c), d, field, c->err);
  int rc = dustb_ghost_add(c, field, 1, stream);
  if (rc) return rc;
  const int nb = 1024;
  k_argmax_blocks<<<nb, 256, 0, S(stream)>>>(d, field, bval, bloc);
  k_argmax_final<<<1, 1, 0, S(stream)>>>(d, mview(c), bval, bloc, nb, row);
  return launch_status("phst");
}

// ---- refinable clouds on a uniform 3-D mesh (periodic; plain P1 hat clouds) ---------------
// (physical x3 faces: the mirrored part of the clouds that reach beyond them; shear-periodic x1
// faces, whose translated parts need the shear images of the neighbours, are not supported)
// (a refined mesh needs the leaf tables; with them a uniform 3-D mesh takes the leaf traversal
// too)
static int cloud_mesh_ok(const dustb_ctx *c) {
  const dustb_mesh &ms = c->mesh;
  if (ms.nghbr_ml || ms.leaf) {
    const dustb_leaf_tables *t = ms.leaf;
    return ms.three_d && !ms.shear_x1 && t && t->fbox && t->blev && t->nnb && t->nb && t->nbs &&
           t->nbmax && t->safe && t->lockey && t->locblk && t->nlev >= 0 && t->nlev <= 16 &&
           t->root_dx[0] > 0.0 && t->root_dx[1] > 0.0 && t->root_dx[2] > 0.0;
  }
  return ms.multi_d && !ms.shear_x1;
}
// the clouds' u* copy exchange: the multilevel one on a refined mesh (leaf->coarse)
static int cloud_ustar_exchange(const dustb_ctx *c, void *stream) {
  if (c->mesh.nghbr_ml)
    return dustb_ghost_copy_ml(c, c->f.ustar, 3, c->mesh.leaf->coarse,
                               c->mesh.leaf->coarse_bytes, stream);
  return dustb_ghost_copy(c, c->f.ustar, 3, 1, stream);
}
static int cloud_x3phys(const dustb_ctx *c) {
  return c->mesh.three_d && c->mesh.x3bc != DUSTB_X3_PERIODIC;
}

long long dustb_cloud_gpack_bytes(const dustb_mesh *mesh) {
  if (!mesh) return -1;
  const Ind d = make_ind(*mesh);
  return n_all(d) * 12 * (long long)sizeof(double);
}

int dustb_cloud_deposit_qp(const dustb_ctx *c, double a_dt, double sh, void *stream) {
  CHECK_CTX(c);
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  const Ind d = make_ind(c->mesh);
  cudaMemsetAsync(c->f.qdep, 0, (size_t)(n_all(d) * 5) * sizeof(double), S(stream));
  if (c->part.npart > 0) {
    if (c->mesh.leaf) k_cloud_deposit_l<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.qdep, a_dt, sh, cloud_x3phys(c), c->err);
    else k_cloud_deposit_u<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.qdep, a_dt, sh, cloud_x3phys(c), c->err);
  }
  return launch_status("cloud_deposit_qp");
}

int dustb_cloud_gather_kick(const dustb_ctx *c, double a_dt, double sh, double *gpack,
                            void *stream) {
  CHECK_CTX(c);
  if (!gpack) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  const Ind d = make_ind(c->mesh);
  k_gather_pack<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(d, c->f.ustar, gpack);
  cudaMemsetAsync(c->f.dmom, 0, (size_t)(n_all(d) * 3) * sizeof(double), S(stream));
  if (c->part.npart > 0) {
    if (c->mesh.leaf) k_cloud_gather_kick_l<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.dmom, a_dt, sh,
                                      c->phys.back_reaction, cloud_x3phys(c), c->err);
    else k_cloud_gather_kick_u<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.dmom, a_dt, sh,
                                      c->phys.back_reaction, cloud_x3phys(c), c->err);
  }
  return launch_status("cloud_gather_kick");
}

int dustb_cloud_dc1_sweep(const dustb_ctx *c, double a_dt, double sh, double *gpack,
                          void *stream) {
  CHECK_CTX(c);
  if (!gpack) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  const Ind d = make_ind(c->mesh);
  int rc = cloud_ustar_exchange(c, stream);
  if (rc) return rc;
  k_gather_pack<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(d, c->f.ustar, gpack);
  cudaMemsetAsync(c->f.work, 0, (size_t)n_all(d) * 3 * sizeof(double), S(stream));
  if (c->part.npart > 0) {
    if (c->mesh.leaf) k_cloud_operator_l<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.work, a_dt, sh,
                                   cloud_x3phys(c), c->err);
    else k_cloud_operator_u<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.work, a_dt, sh,
                                   cloud_x3phys(c), c->err);
  }
  k_dc_correct<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(d, c->f.u0, c->f.nvar_gas,
                                                                    c->f.qdep, c->f.work,
                                                                    c->f.ustar);
  return launch_status("cloud_dc1_sweep");
}

int dustb_cloud_apply_pmbr(const dustb_ctx *c, double a_dt, double sh, void *stream) {
  CHECK_CTX(c);
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  if (!c->phys.back_reaction) return DUSTB_OK;
  if (!c->phys.consistent_gas) return dustb_apply_pmbr(c, a_dt, stream);
  const Ind d = make_ind(c->mesh);
  cudaMemsetAsync(c->f.resid, 0, (size_t)n_all(d) * 4 * sizeof(double), S(stream));
  k_cloud_consistent_gas<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(
      d, c->f.u0, c->f.nvar_gas, c->f.ustar, c->f.qdep, c->f.dmom, c->f.resid, 1.0 / a_dt);
  if (c->part.npart > 0) {
    if (c->mesh.leaf) k_cloud_consistent_dust_l<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.resid, a_dt, sh,
                                          cloud_x3phys(c));
    else k_cloud_consistent_dust_u<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.resid, a_dt, sh,
                                          cloud_x3phys(c));
  }
  return launch_status("cloud_apply_pmbr");
}

int dustb_cloud_pc2_predictor(const dustb_ctx *c, double dt, int rate_dep, double *gpack,
                              void *stream) {
  CHECK_CTX(c);
  if (!gpack) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  const Ind d = make_ind(c->mesh);
  cudaMemsetAsync(c->f.qdep, 0, (size_t)(n_all(d) * 5) * sizeof(double), S(stream));
  // the step-start gas velocity in work, packed with its central differences
  k_gas_velocity_all<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(d, c->f.u1, c->f.nvar_gas,
                                                                        c->f.work);
  k_gather_pack<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(d, c->f.work, gpack);
  if (c->part.npart > 0) {
    if (c->mesh.leaf) k_cloud_pc2_predictor_l<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.qdep, dt, rate_dep,
                                        cloud_x3phys(c), c->err);
    else k_cloud_pc2_predictor_u<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.qdep, dt, rate_dep,
                                        cloud_x3phys(c), c->err);
  }
  return launch_status("cloud_pc2_predictor");
}

int dustb_cloud_pc2_advance(const dustb_ctx *c, double dt, double *gpack, void *stream) {
  CHECK_CTX(c);
  if (!gpack) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  const Ind d = make_ind(c->mesh);
  const dustb_physics &ph = c->phys;
  k_gather_pack<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(d, c->f.ustar, gpack);
  cudaMemsetAsync(c->f.dmom, 0, (size_t)(n_all(d) * 3) * sizeof(double), S(stream));
  if (c->part.npart > 0) {
    if (c->mesh.leaf) k_cloud_pc2_advance_l<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.dmom, dt,
                                      ph.back_reaction, ph.shearing_box, ph.stratified,
                                      ph.qshear, ph.omega0, ph.const_accel_phi, cloud_x3phys(c), c->err);
    else k_cloud_pc2_advance_u<<<PGRID(c)>>>(pview(c), mview(c), d, gpack, c->f.dmom, dt,
                                      ph.back_reaction, ph.shearing_box, ph.stratified,
                                      ph.qshear, ph.omega0, ph.const_accel_phi, cloud_x3phys(c), c->err);
  }
  return launch_status("cloud_pc2_advance");
}

// ---- cloud management on a refined mesh: the instant switch and the P1 split -------------
int dustb_cloud_instant_switch(const dustb_ctx *c, int level_cap, int *nchange, void *scratch,
                               void *stream) {
  CHECK_CTX(c);
  if (!nchange || !scratch) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c) || !c->mesh.leaf) return DUSTB_EUNSUP;
  *nchange = 0;
  if (level_cap < 0 || level_cap >= c->mesh.leaf->nlev || c->part.npart == 0) return DUSTB_OK;
  const Ind d = make_ind(c->mesh);
  int *cnt = (int *)scratch;
  cudaMemsetAsync(cnt, 0, sizeof(int), S(stream));
  k_cloud_instant_switch<<<PGRID(c)>>>(pview(c), mview(c), d, level_cap, cnt);
  int rc = launch_status("cloud_instant_switch");
  if (rc) return rc;
  cudaMemcpyAsync(nchange, cnt, sizeof(int), cudaMemcpyDeviceToHost, S(stream));
  cudaStreamSynchronize(S(stream));
  return launch_status("cloud_instant_switch");
}

long long dustb_cloud_split_scratch_bytes(int npart) {
  if (npart < 0) return -1;
  const long long n = (long long)npart + 1;
  return ((2 * n * 4 + 255) & ~255LL) + ((scan_bsum_ints(n) * 4 + 255) & ~255LL) + 256;
}

int dustb_cloud_split_p1(const dustb_ctx *c, const dustb_cloud_split *sp,
                         unsigned long long tag0, int *nnew, void *scratch, long long bytes,
                         void *stream) {
  CHECK_CTX(c);
  if (!sp || !nnew || !(sp->slack >= 0.0 && sp->slack < 1.0) || sp->split_buffer < 0 ||
      sp->budget < 0)
    return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c) || !c->mesh.leaf) return DUSTB_EUNSUP;
  *nnew = 0;
  const int np = c->part.npart;
  if (np == 0) return DUSTB_OK;
  if (!scratch || bytes < dustb_cloud_split_scratch_bytes(np)) return DUSTB_ESCRATCH;
  const Ind d = make_ind(c->mesh);
  SplitCtl C{};
  C.max_level = sp->max_level;
  C.everywhere = sp->split_everywhere;
  C.overlap = sp->split_overlap;
  C.slack = sp->slack;
  const int nlev = c->mesh.leaf->nlev;
  for (int l = 0; l <= 17; ++l)
    C.rdil[l] = (sp->split_buffer > 0 && l >= 1 && l <= nlev) ? (sp->split_buffer << (nlev - l + 1))
                                                             : 0;
  const long long n1 = (long long)np + 1;
  int *off = (int *)scratch;
  int *sep = off + n1;
  int *bsum = (int *)((char *)scratch + ((2 * n1 * 4 + 255) & ~255LL));
  int *taken = (int *)((char *)bsum + ((scan_bsum_ints(n1) * 4 + 255) & ~255LL));
  cudaMemsetAsync(off + np, 0, sizeof(int), S(stream));
  k_split_count<<<PGRID(c)>>>(pview(c), mview(c), d, C, off, sep);
  int rc = launch_status("cloud_split_p1");
  if (rc) return rc;
  rc = exclusive_scan(off, n1, bsum, S(stream));
  if (rc) return rc;
  int total = 0;
  cudaMemcpyAsync(&total, off + np, sizeof(int), cudaMemcpyDeviceToHost, S(stream));
  cudaStreamSynchronize(S(stream));
  rc = launch_status("cloud_split_p1");
  if (rc) return rc;
  if (sp->budget > 0 && (long long)total > sp->budget) {
    // the events beyond the budget wait; the pieces of those taken
    cudaMemcpyAsync(taken, off + np, sizeof(int), cudaMemcpyDeviceToDevice, S(stream));
    k_split_budget<<<PGRID(c)>>>(sep, off, np, sp->budget, taken);
    cudaMemcpyAsync(&total, taken, sizeof(int), cudaMemcpyDeviceToHost, S(stream));
    cudaStreamSynchronize(S(stream));
    rc = launch_status("cloud_split_p1");
    if (rc) return rc;
  }
  *nnew = total;
  if ((long long)np + total > c->part.stride) {
    dustb_host::set_message("cloud_split_p1: the pieces exceed the particle capacity");
    return DUSTB_ESCRATCH;
  }
  const int x3reflect = c->mesh.three_d && c->mesh.x3bc == DUSTB_X3_REFLECT;
  k_split_fill<<<PGRID(c)>>>(pview(c), mview(c), d, sep, off, tag0, np, x3reflect);
  return launch_status("cloud_split_p1");
}

// the point transfers' remap: the drag's, with the ghost deposits behind physical x3 faces
// always folded (src/dust/dust_gravity_points.cpp:176-178)
static dustb_ctx fold_ctx(const dustb_ctx *c) {
  dustb_ctx g = *c;
  g.phys.x3_deposit_drop = 0;
  return g;
}

static int point_deposit(const dustb_ctx *c, double *out, double *halo, int ncomp, int species,
                         int gravity, void *stream) {
  const Ind d = make_ind(c->mesh);
  const dustb_ctx g = fold_ctx(c);
  cudaMemsetAsync(halo, 0, (size_t)(n_all(d) * ncomp) * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_point_deposit<<<PGRID(c)>>>(pview(c), mview(c), d, halo, ncomp, species, gravity, c->err);
  int rc = dustb_ghost_add(&g, halo, ncomp, stream);
  if (rc) return rc;
  k_owned_copy<<<blocks_for(n_all(d) * ncomp), kThreads, 0, S(stream)>>>(d, halo, out, ncomp);
  return launch_status("point_deposit");
}

int dustb_point_gravity_density(const dustb_ctx *c, double *owned, double *halo, void *stream) {
  CHECK_CTX(c);
  if (!owned || !halo) return DUSTB_EINVAL;
  if (!c->mesh.three_d || c->phys.scheme != DUSTB_TSC) return DUSTB_EUNSUP;
  return point_deposit(c, owned, halo, 1, -1, 1, stream);
}

int dustb_point_science_fields(const dustb_ctx *c, double *out, double *halo, int mass_only,
                               int species, void *stream) {
  CHECK_CTX(c);
  if (!out || !halo) return DUSTB_EINVAL;
  if (!c->mesh.three_d) return DUSTB_EUNSUP;
  return point_deposit(c, out, halo, mass_only ? 1 : 4, species, 0, stream);
}

int dustb_point_gravity_gather(const dustb_ctx *c, const double *owned, double *halo,
                               double *acc, long long acc_stride, void *stream) {
  CHECK_CTX(c);
  if (!owned || !halo || !acc || acc_stride < c->part.npart) return DUSTB_EINVAL;
  if (!c->mesh.three_d || c->phys.scheme != DUSTB_TSC) return DUSTB_EUNSUP;
  const Ind d = make_ind(c->mesh);
  const dustb_ctx g = fold_ctx(c);
  const SBox B = sbview(&g);
  if (B.on && (!B.sb_gid || B.nb2 <= 0 || B.nb3 <= 0)) return DUSTB_EINVAL;
  k_point_force_field<<<blocks_for(n_all(d)), kThreads, 0, S(stream)>>>(
      d, c->mesh.nghbr, c->mesh.gids, B, owned, halo, 3);
  if (c->part.npart > 0)
    k_point_gather<<<PGRID(c)>>>(pview(c), mview(c), d, halo, acc, acc_stride, c->err);
  return launch_status("point_gravity_gather");
}

// one imex2+ cycle in the task order of src/dust/dust_tasks.cpp:38-120 (stage 3 dormant,
// dust.cpp:1646-1649); tableau src/driver/driver.cpp:278-300
int dustb_imex_cycle(const dustb_ctx *c, const dustb_imex_coeffs *co, double *x3_removed,
                     void *stream) {
  CHECK_CTX(c);
  if (!co || !(co->dt > 0.0)) return DUSTB_EINVAL;
  const double g = co->gamma, dt = co->dt;
  const double gam0[2] = {1.0, (2.0 * g - 1.0) / (2.0 * g * g)};
  const double gam1[2] = {0.0, 1.0 - (2.0 * g - 1.0) / (2.0 * g * g)};
  const double beta[2] = {g, 1.0 / (2.0 * g)};
  const double atw22 = (1.0 - 2.0 * g * g) / 2.0 / g;
  const double a_dt = g * dt;
  const int br = c->phys.back_reaction;
  int rc;
#define RUN(x) do { rc = (x); if (rc) return rc; } while (0)
  for (int stage = 1; stage <= 2; ++stage) {
    if (stage == 1) RUN(dustb_register_copy(c, stream));
    RUN(dustb_gas_rk_noflux(c, gam0[stage - 1], gam1[stage - 1], stream));
    if (stage == 2 && br) RUN(dustb_history_gas(c, atw22 * dt, stream));
    RUN(dustb_push_imex(c, gam0[stage - 1], gam1[stage - 1], beta[stage - 1] * dt,
                        (stage == 2) ? atw22 * dt : 0.0, stream));
    RUN(dustb_route(c, x3_removed, stream));
    const double sh = co->sh[stage - 1];
    if (br) {
      RUN(dustb_deposit_qp(c, a_dt, sh, stream));
      RUN(dustb_ghost_add(c, c->f.qdep, 5, stream));
    }
    RUN(dustb_solve_ustar(c, stream));
    if (br && c->phys.drag_solver >= DUSTB_SOLVER_DC1) {
      int nsw = (c->phys.drag_solver == DUSTB_SOLVER_DC2) ? 2 : 1;
      for (int w = 0; w < nsw; ++w) RUN(dustb_dc1_sweep(c, a_dt, sh, stream));
    }
    RUN(dustb_ghost_copy(c, c->f.ustar, 3, 1, stream));
    RUN(dustb_gather_kick_pmbr(c, a_dt, sh, stream));
    if (br) {
      RUN(dustb_ghost_add(c, c->f.dmom, 3, stream));
      RUN(dustb_apply_pmbr(c, a_dt, stream));
    }
    RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, stream));
  }
  return DUSTB_OK;
}

// one imex2+ cycle on a refined mesh: the task order of dustb_imex_cycle with the deposits
// exchanged by the general remap and u*, the operator's field and the gas state by the
// multilevel copy exchange
// ApplyDefectCorrection (dust_solver.cpp:226-252), one sweep on a refined mesh: u*'s ghost
// cells by the multilevel copy exchange, the operator's ghost deposits by the general remap
int dustb_dc1_sweep_plan(const dustb_ctx *c, const dustb_dep_plan *plan, double a_dt,
                         double *coarse, long long coarse_bytes, void *stream) {
  CHECK_CTX(c);
  if (!plan || !c->mesh.nghbr_ml) return DUSTB_EINVAL;
  const Ind d = make_ind(c->mesh);
  int rc = dustb_ghost_copy_ml(c, c->f.ustar, 3, coarse, coarse_bytes, stream);
  if (rc) return rc;
  cudaMemsetAsync(c->f.work, 0, (size_t)n_all(d) * 3 * sizeof(double), S(stream));
  if (c->part.npart > 0)
    k_operator<<<PGRID(c)>>>(pview(c), mview(c), d, c->f.ustar, c->f.work, a_dt, 0.0, c->err);
  rc = dustb_ghost_add_plan(c, plan, c->f.work, 3, stream);
  if (rc) return rc;
  k_dc_correct<<<blocks_for(n_active(d)), kThreads, 0, S(stream)>>>(
      d, c->f.u0, c->f.nvar_gas, c->f.qdep, c->f.work, c->f.ustar);
  return launch_status("dc1_sweep_plan");
}

int dustb_refined_imex_cycle(const dustb_ctx *c, const dustb_dep_plan *plan,
                             const dustb_imex_coeffs *co, double *coarse, long long coarse_bytes,
                             double *x3_removed, void *stream) {
  CHECK_CTX(c);
  if (!co || !(co->dt > 0.0) || !plan || !c->mesh.nghbr_ml) return DUSTB_EINVAL;
  if (co->sh[0] != 0.0 || co->sh[1] != 0.0) return DUSTB_EUNSUP;    // (no shearing box)
  const double g = co->gamma, dt = co->dt;
  const double gam0[2] = {1.0, (2.0 * g - 1.0) / (2.0 * g * g)};
  const double gam1[2] = {0.0, 1.0 - (2.0 * g - 1.0) / (2.0 * g * g)};
  const double beta[2] = {g, 1.0 / (2.0 * g)};
  const double atw22 = (1.0 - 2.0 * g * g) / 2.0 / g;
  const double a_dt = g * dt;
  const int br = c->phys.back_reaction;
  Ind d = make_ind(c->mesh);
  int rc;
  for (int stage = 1; stage <= 2; ++stage) {
    if (stage == 1) RUN(dustb_register_copy(c, stream));
    RUN(dustb_gas_rk_noflux(c, gam0[stage - 1], gam1[stage - 1], stream));
    if (stage == 2 && br) RUN(dustb_history_gas(c, atw22 * dt, stream));
    RUN(dustb_push_imex(c, gam0[stage - 1], gam1[stage - 1], beta[stage - 1] * dt,
                        (stage == 2) ? atw22 * dt : 0.0, stream));
    RUN(dustb_route(c, x3_removed, stream));
    if (br) {
      RUN(dustb_deposit_qp(c, a_dt, 0.0, stream));
      RUN(dustb_ghost_add_plan(c, plan, c->f.qdep, 5, stream));
    }
    RUN(dustb_solve_ustar(c, stream));
    if (br && c->phys.drag_solver >= DUSTB_SOLVER_DC1) {
      const int nsw = (c->phys.drag_solver == DUSTB_SOLVER_DC2) ? 2 : 1;
      for (int w = 0; w < nsw; ++w)
        RUN(dustb_dc1_sweep_plan(c, plan, a_dt, coarse, coarse_bytes, stream));
    }
    RUN(dustb_ghost_copy_ml(c, c->f.ustar, 3, coarse, coarse_bytes, stream));
    RUN(dustb_gather_kick_pmbr(c, a_dt, 0.0, stream));
    if (br) {
      RUN(dustb_ghost_add_plan(c, plan, c->f.dmom, 3, stream));
      RUN(dustb_apply_pmbr(c, a_dt, stream));
    }
    RUN(dustb_ghost_copy_ml(c, c->f.u0, c->f.nvar_gas, coarse, coarse_bytes, stream));
  }
  return launch_status("refined_imex_cycle");
}

// one imex2+ cycle of refinable clouds on a uniform mesh: the task order of dustb_imex_cycle
// with the clouds' deposit (into the owner cells: no deposit exchange), dc1 / dc2 sweeps,
// gather-kick and PMBR split
static int cloud_imex_cycle(const dustb_ctx *c, const dustb_imex_coeffs *co, double *gpack,
                            double *coarse, long long coarse_bytes, double *x3_removed,
                            void *stream) {
  // the gas state's copy exchange: the multilevel one on a refined mesh
  auto gas_exchange = [&]() {
    return c->mesh.nghbr_ml
               ? dustb_ghost_copy_ml(c, c->f.u0, c->f.nvar_gas, coarse, coarse_bytes, stream)
               : dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, stream);
  };
  const double g = co->gamma, dt = co->dt;
  const double gam0[2] = {1.0, (2.0 * g - 1.0) / (2.0 * g * g)};
  const double gam1[2] = {0.0, 1.0 - (2.0 * g - 1.0) / (2.0 * g * g)};
  const double beta[2] = {g, 1.0 / (2.0 * g)};
  const double atw22 = (1.0 - 2.0 * g * g) / 2.0 / g;
  const double a_dt = g * dt;
  const int br = c->phys.back_reaction;
  int rc;
  for (int stage = 1; stage <= 2; ++stage) {
    if (stage == 1) RUN(dustb_register_copy(c, stream));
    RUN(dustb_gas_rk_noflux(c, gam0[stage - 1], gam1[stage - 1], stream));
    if (stage == 2 && br) RUN(dustb_history_gas(c, atw22 * dt, stream));
    RUN(dustb_push_imex(c, gam0[stage - 1], gam1[stage - 1], beta[stage - 1] * dt,
                        (stage == 2) ? atw22 * dt : 0.0, stream));
    RUN(dustb_route(c, x3_removed, stream));
    const double sh = co->sh[stage - 1];
    if (br) RUN(dustb_cloud_deposit_qp(c, a_dt, sh, stream));
    RUN(dustb_solve_ustar(c, stream));
    if (br && c->phys.drag_solver >= DUSTB_SOLVER_DC1) {
      int nsw = (c->phys.drag_solver == DUSTB_SOLVER_DC2) ? 2 : 1;
      for (int w = 0; w < nsw; ++w) RUN(dustb_cloud_dc1_sweep(c, a_dt, sh, gpack, stream));
    }
    RUN(cloud_ustar_exchange(c, stream));
    RUN(dustb_cloud_gather_kick(c, a_dt, sh, gpack, stream));
    if (br) RUN(dustb_cloud_apply_pmbr(c, a_dt, sh, stream));
    RUN(gas_exchange());
  }
  return DUSTB_OK;
}

int dustb_cloud_imex_cycle(const dustb_ctx *c, const dustb_imex_coeffs *co, double *gpack,
                           double *x3_removed, void *stream) {
  CHECK_CTX(c);
  if (!co || !(co->dt > 0.0) || !gpack) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c) || c->mesh.nghbr_ml) return DUSTB_EUNSUP;
  return cloud_imex_cycle(c, co, gpack, nullptr, 0, x3_removed, stream);
}

int dustb_cloud_refined_imex_cycle(const dustb_ctx *c, const dustb_imex_coeffs *co,
                                   double *gpack, double *coarse, long long coarse_bytes,
                                   double *x3_removed, void *stream) {
  CHECK_CTX(c);
  if (!co || !(co->dt > 0.0) || !gpack || !c->mesh.leaf) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  if (co->sh[0] != 0.0 || co->sh[1] != 0.0) return DUSTB_EUNSUP;    // (no shearing box)
  return cloud_imex_cycle(c, co, gpack, coarse, coarse_bytes, x3_removed, stream);
}

// one pc2 cycle of the clouds: the order of dustb_pc2_cycle with the clouds' predictor and
// advance (their deposits in the owner cells: no deposit exchanges)
int dustb_cloud_pc2_cycle(const dustb_ctx *c, double dt, double *chi_max, double *gpack,
                          double *x3_removed, void *stream) {
  CHECK_CTX(c);
  if (!(dt > 0.0) || !gpack) return DUSTB_EINVAL;
  if (!cloud_mesh_ok(c)) return DUSTB_EUNSUP;
  const int br = c->phys.back_reaction;
  int rc;
  RUN(dustb_register_copy(c, stream));
  RUN(dustb_gas_rk_noflux(c, 1.0, 0.0, stream));
  if (br) {
    RUN(dustb_cloud_pc2_predictor(c, dt, 1, gpack, stream));
    RUN(dustb_pc2_apply_predictor(c, dt, chi_max, stream));
  }
  RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, stream));
  RUN(dustb_pc2_midpoint(c, stream));
  RUN(dustb_gas_rk_noflux(c, 0.5, 0.5, stream));
  RUN(dustb_cloud_pc2_advance(c, dt, gpack, stream));
  RUN(dustb_route(c, x3_removed, stream));
  if (br) RUN(dustb_pc2_commit(c, 0.5, stream));
  RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, stream));
  return DUSTB_OK;
}

// one pc2 cycle (integrator rk2): stage 1 predictor, stage 2 midpoint advance and commit
int dustb_pc2_cycle(const dustb_ctx *c, double dt, double *chi_max, double *x3_removed,
                    void *stream) {
  CHECK_CTX(c);
  if (!(dt > 0.0)) return DUSTB_EINVAL;
  const int br = c->phys.back_reaction;
  int rc;
  RUN(dustb_register_copy(c, stream));
  RUN(dustb_gas_rk_noflux(c, 1.0, 0.0, stream));
  if (br) {
    RUN(dustb_pc2_predictor(c, dt, 1, stream));
    RUN(dustb_ghost_add(c, c->f.qdep, 5, stream));
    RUN(dustb_pc2_apply_predictor(c, dt, chi_max, stream));
  }
  RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, stream));
  RUN(dustb_pc2_midpoint(c, stream));
  RUN(dustb_gas_rk_noflux(c, 0.5, 0.5, stream));
  RUN(dustb_pc2_advance(c, dt, stream));
  RUN(dustb_route(c, x3_removed, stream));
  if (br) {
    RUN(dustb_ghost_add(c, c->f.dmom, 3, stream));
    RUN(dustb_pc2_commit(c, 0.5, stream));
  }
  RUN(dustb_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0, stream));
#undef RUN
  return DUSTB_OK;
}

}  // extern "C"
