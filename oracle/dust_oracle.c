/*
 * dust_oracle.c -- CPU oracle of the dust particle-drag step.  TEST INFRASTRUCTURE ONLY:
 * the tests, the smoke check and the CPU-baseline leg of the benchmark call it as the
 * checker; the product path (athenak_b200) never links or calls it.
 *
 * A plain-C FP64 restatement of the reference kernels, function by function, in the
 * reference's data layout (dustb.h).  Each function names the file:line it follows.  The
 * loops run in the reference's iteration order; with one thread the deposits are plain
 * sums in particle order (Kokkos Serial's DepositAdd, src/dust/dust.hpp:986-998); with
 * OpenMP threads they are atomic adds (the Kokkos OpenMP backend), which is the form timed
 * as the CPU baseline.
 *
 * Parity pins: the reference ships no golden output files and its Kokkos build cannot be
 * compiled here (the kokkos submodule is empty), so the oracle is pinned to the
 * reference's own known-answer tests instead: the dust_damping ODE
 * (src/pgen/tests/dust_damping.cpp:9-16), exact total-momentum conservation
 * (tst/test_suite/dust/check_cloud_imex3d.py:66-74) and the NSH drift
 * (src/pgen/dust_amr/dust_setup.hpp:58-65); see tests/test_oracle_kat.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/dustb.h"

#define SQR(x) ((x)*(x))

static int g_threads = 1;
void oracle_set_threads(int n) { g_threads = (n < 1) ? 1 : n; }
int oracle_get_threads(void) { return g_threads; }

/* ---- layout helpers ------------------------------------------------------------------ */
typedef struct {
  int n1, n2, n3, is, ie, js, je, ks, ke;
} Ind;

static Ind indices(const dustb_mesh *ms) {
  Ind d;
  d.n1 = ms->nx1 + 2*ms->ng;
  d.n2 = ms->multi_d ? ms->nx2 + 2*ms->ng : 1;
  d.n3 = ms->three_d ? ms->nx3 + 2*ms->ng : 1;
  d.is = ms->ng; d.ie = d.is + ms->nx1 - 1;
  d.js = ms->multi_d ? ms->ng : 0; d.je = d.js + (ms->multi_d ? ms->nx2 : 1) - 1;
  d.ks = ms->three_d ? ms->ng : 0; d.ke = d.ks + (ms->three_d ? ms->nx3 : 1) - 1;
  return d;
}

#define A5(arr, nv, d, m, v, k, j, i) \
  (arr)[((((size_t)(m)*(nv) + (v))*(d).n3 + (k))*(d).n2 + (j))*(d).n1 + (i)]
#define PR(c, p) pr[(size_t)(c)*stride + (p)]
#define PI(c, p) pi[(size_t)(c)*stride + (p)]
#define MB(m, f) ms->mb_size[(size_t)(m)*9 + (f)]
enum { X1MIN = 0, X2MIN = 1, X3MIN = 2, X1MAX = 3, X2MAX = 4, X3MAX = 5, DX1 = 6, DX2 = 7,
       DX3 = 8 };

static inline void deposit_add(double *dst, double v) {
#pragma omp atomic
  *dst += v;
}

/* PMWeights, src/dust/dust.hpp:1088-1111 */
static inline void pm_weights(double x, double xmin, double xmax, int nx, int is, int scheme,
                              int *ip, double w[3]) {
  double cell = (x - xmin)*((double)nx/(xmax - xmin));
  int ig = (int)(cell + 1.0) - 1;
  double del = cell - ((double)ig + 0.5);
  *ip = ig + is;
  if (scheme == 0) {
    w[0] = 0.0; w[1] = 1.0; w[2] = 0.0;
  } else if (scheme == 1) {
    w[0] = fmax(0.0, -del); w[1] = 1.0 - fabs(del); w[2] = fmax(0.0, del);
  } else {
    w[0] = 0.5*SQR(0.5 - del); w[1] = 0.75 - SQR(del); w[2] = 0.5*SQR(0.5 + del);
  }
}

/* the three weight sets of particle p at (x, y + sh x, z) */
static inline void particle_weights(const dustb_ctx *c, const Ind *d, int m, double x,
                                    double y, double z, int *ip, int *jp, int *kp,
                                    double wx[3], double wy[3], double wz[3]) {
  const dustb_mesh *ms = &c->mesh;
  int sch = c->phys.scheme;
  pm_weights(x, MB(m, X1MIN), MB(m, X1MAX), ms->nx1, d->is, sch, ip, wx);
  pm_weights(y, MB(m, X2MIN), MB(m, X2MAX), ms->nx2, d->js, sch, jp, wy);
  if (ms->three_d) {
    pm_weights(z, MB(m, X3MIN), MB(m, X3MAX), ms->nx3, d->ks, sch, kp, wz);
  } else {
    *kp = d->ks; wz[0] = 0.0; wz[1] = 1.0; wz[2] = 0.0;
  }
}

static inline double cell_volume(const dustb_mesh *ms, int m) {
  double vol = MB(m, DX1)*MB(m, DX2);
  if (ms->three_d) vol *= MB(m, DX3);
  return vol;
}

static int halo_ok(const dustb_mesh *ms, const Ind *d, int ip, int jp, int kp) {
  if (ip < d->is - 1 || ip > d->is + ms->nx1) return 0;
  if (jp < d->js - 1 || jp > d->js + ms->nx2) return 0;
  if (ms->three_d && (kp < d->ks - 1 || kp > d->ks + ms->nx3)) return 0;
  return 1;
}

static size_t field_size(const dustb_mesh *ms, int nvar) {
  Ind d = indices(ms);
  return (size_t)ms->nmb*nvar*d.n3*d.n2*d.n1;
}

/* ---- FirstTwoImpRK stage 1, src/dust/dust_push.cpp:63-79 ------------------------------ */
void oracle_register_copy(const dustb_ctx *c) {
  const dustb_mesh *ms = &c->mesh;
  memcpy(c->f.u1, c->f.u0, field_size(ms, c->f.nvar_gas)*sizeof(double));
  double *pr = c->part.pr; long long stride = c->part.stride;
  for (int p = 0; p < c->part.npart; ++p) {
    PR(DUSTB_IPX1, p) = PR(DUSTB_IPX, p);
    PR(DUSTB_IPVX1, p) = PR(DUSTB_IPVX, p);
    PR(DUSTB_IPY1, p) = PR(DUSTB_IPY, p);
    PR(DUSTB_IPVY1, p) = PR(DUSTB_IPVY, p);
    PR(DUSTB_IPZ1, p) = PR(DUSTB_IPZ, p);
    PR(DUSTB_IPVZ1, p) = PR(DUSTB_IPVZ, p);
  }
}

/* stand-in for Hydro::RKUpdate with a zero flux divergence (active cells) */
void oracle_gas_rk_noflux(const dustb_ctx *c, double gam0, double gam1) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  for (int m = 0; m < ms->nmb; ++m)
    for (int v = 0; v < nv; ++v)
      for (int k = d.ks; k <= d.ke; ++k)
        for (int j = d.js; j <= d.je; ++j)
          for (int i = d.is; i <= d.ie; ++i)
            A5(c->f.u0, nv, d, m, v, k, j, i) = gam0*A5(c->f.u0, nv, d, m, v, k, j, i) +
                                                gam1*A5(c->f.u1, nv, d, m, v, k, j, i);
}

/* AddDragHistoryGas, src/dust/dust_pm.cpp:721-742 */
void oracle_history_gas(const dustb_ctx *c, double atw_dt) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i)
          for (int v = 0; v < 3; ++v)
            A5(c->f.u0, nv, d, m, 1 + v, k, j, i) += atw_dt*A5(c->f.dmom, 3, d, m, v, k, j, i);
}

/* ExplicitPush imex branch, src/dust/dust_push.cpp:249-297 */
void oracle_push_imex(const dustb_ctx *c, double gam0, double gam1, double beta_dt,
                      double atw_dt) {
  double *pr = c->part.pr; long long stride = c->part.stride;
  const int three_d = c->mesh.three_d, sbox = c->phys.shearing_box, strat = c->phys.stratified;
  const double q = c->phys.qshear, om = c->phys.omega0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int p = 0; p < c->part.npart; ++p) {
    double x_old = PR(DUSTB_IPX, p), y_old = PR(DUSTB_IPY, p), z_old = PR(DUSTB_IPZ, p);
    double vx_old = PR(DUSTB_IPVX, p), vy_old = PR(DUSTB_IPVY, p), vz_old = PR(DUSTB_IPVZ, p);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    if (sbox) {
      if (three_d) {
        fx = 2.0*om*vy_old;
        fy = -(2.0 - q)*om*vx_old;
        if (strat) fz = -SQR(om)*z_old;
      } else {
        fx = 2.0*om*vz_old;
        fz = -(2.0 - q)*om*vx_old;
      }
    }
    PR(DUSTB_IPVX, p) = gam0*vx_old + gam1*PR(DUSTB_IPVX1, p) + beta_dt*fx + atw_dt*PR(DUSTB_IPRX, p);
    PR(DUSTB_IPVY, p) = gam0*vy_old + gam1*PR(DUSTB_IPVY1, p) + beta_dt*fy + atw_dt*PR(DUSTB_IPRY, p);
    PR(DUSTB_IPVZ, p) = gam0*vz_old + gam1*PR(DUSTB_IPVZ1, p) + beta_dt*fz + atw_dt*PR(DUSTB_IPRZ, p);
    double ydot = vy_old;
    if (sbox && three_d) ydot -= q*om*x_old;
    PR(DUSTB_IPX, p) = gam0*x_old + gam1*PR(DUSTB_IPX1, p) + beta_dt*vx_old;
    PR(DUSTB_IPY, p) = gam0*y_old + gam1*PR(DUSTB_IPY1, p) + beta_dt*ydot;
    if (three_d) PR(DUSTB_IPZ, p) = gam0*z_old + gam1*PR(DUSTB_IPZ1, p) + beta_dt*vz_old;
  }
}

/* SetNewPrtclGID, src/bvals/bvals_part.cpp:115-429, single-level mesh (shear-periodic x1 faces
 * :133-141, :266-310).  Returns the OR of the error bits of the particles it could not route. */
unsigned oracle_route(const dustb_ctx *c, double *x3_removed) {
  const dustb_mesh *ms = &c->mesh;
  double *pr = c->part.pr; int *pi = c->part.pi; long long stride = c->part.stride;
  unsigned err = 0;
  const double z3a = ms->x3min, z3b = ms->x3max;
  const int shear_x1 = ms->shear_x1 && ms->three_d;
  double ysh = 0.0;
  if (shear_x1) {
    const double lxm = ms->x1max - ms->x1min, lym = ms->x2max - ms->x2min;
    ysh = fmod(c->phys.qshear*c->phys.omega0*lxm*(ms->time), lym);
  }
  for (int p = 0; p < c->part.npart; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    if (m < 0 || m >= ms->nmb) { err |= DUSTB_ERR_PGID; continue; }
    if (ms->x3bc != 0 && (PR(DUSTB_IPZ, p) < z3a || PR(DUSTB_IPZ, p) >= z3b)) {
      const int lo = (PR(DUSTB_IPZ, p) < z3a);
      if (ms->x3bc == 1) {
        const double zf = lo ? z3a : z3b;
        double z = 2.0*zf - PR(DUSTB_IPZ, p);
        if (z >= z3b) z = z3b - 1.0e-12*(z3b - z3a);
        if (z < z3a) z = z3a;
        PR(DUSTB_IPZ, p) = z;
        PR(DUSTB_IPVZ, p) = -PR(DUSTB_IPVZ, p);
        PR(DUSTB_IPZ1, p) = 2.0*zf - PR(DUSTB_IPZ1, p);
        PR(DUSTB_IPVZ1, p) = -PR(DUSTB_IPVZ1, p);
      } else {
        if (x3_removed) { x3_removed[0] += PR(DUSTB_IPM, p); x3_removed[1] += 1.0; }
        PR(DUSTB_IPM, p) = 0.0;
        const double dz = MB(m, DX3);
        const double z = lo ? (MB(m, X3MIN) + 0.5*dz) : (MB(m, X3MAX) - 0.5*dz);
        PR(DUSTB_IPZ, p) = z;
        PR(DUSTB_IPVX, p) = 0.0; PR(DUSTB_IPVY, p) = 0.0; PR(DUSTB_IPVZ, p) = 0.0;
        PR(DUSTB_IPX1, p) = PR(DUSTB_IPX, p); PR(DUSTB_IPY1, p) = PR(DUSTB_IPY, p);
        PR(DUSTB_IPZ1, p) = z;
        PR(DUSTB_IPVX1, p) = 0.0; PR(DUSTB_IPVY1, p) = 0.0; PR(DUSTB_IPVZ1, p) = 0.0;
      }
    }
    double x1 = PR(DUSTB_IPX, p), x2 = PR(DUSTB_IPY, p), x3 = PR(DUSTB_IPZ, p);
    const double lx = MB(m, X1MAX) - MB(m, X1MIN);
    const double ly = MB(m, X2MAX) - MB(m, X2MIN);
    const double lz = MB(m, X3MAX) - MB(m, X3MIN);
    int ix = (int)((x1 - MB(m, X1MIN) + lx)/lx) - 1;
    int iy = (int)((x2 - MB(m, X2MIN) + ly)/ly) - 1;
    int iz = (int)((x3 - MB(m, X3MIN) + lz)/lz) - 1;
    /* snap (bvals_part.cpp:230-247) */
#define SNAP(off, x, xa, xb, ipx, irx) do { \
      if ((off) == 0) { double xs = (x); \
        if ((x) < (xa)) xs = (xa); else if ((x) >= (xb)) xs = nextafter((xb), (xa)); \
        if (xs != (x)) { PR(irx, p) += xs - (x); PR(ipx, p) = xs; (x) = xs; } } } while (0)
    SNAP(ix, x1, MB(m, X1MIN), MB(m, X1MAX), DUSTB_IPX, DUSTB_IPX1);
    if (ms->multi_d) SNAP(iy, x2, MB(m, X2MIN), MB(m, X2MAX), DUSTB_IPY, DUSTB_IPY1);
    if (ms->three_d) SNAP(iz, x3, MB(m, X3MIN), MB(m, X3MAX), DUSTB_IPZ, DUSTB_IPZ1);
#undef SNAP
    if (!ms->multi_d) iy = 0;
    if (!ms->three_d) iz = 0;
    if (abs(ix) > 1 || abs(iy) > 1 || abs(iz) > 1) { err |= DUSTB_ERR_ROUTE; continue; }
    if (ix == 0 && iy == 0 && iz == 0) continue;
    const int lo1 = (ix < 0) && (MB(m, X1MIN) < ms->x1min + 0.5*lx);
    const int hi1 = (ix > 0) && (MB(m, X1MAX) > ms->x1max - 0.5*lx);
    const int lo2 = (iy < 0) && (MB(m, X2MIN) < ms->x2min + 0.5*ly);
    const int hi2 = (iy > 0) && (MB(m, X2MAX) > ms->x2max - 0.5*ly);
    const int lo3 = (iz < 0) && (MB(m, X3MIN) < ms->x3min + 0.5*lz);
    const int hi3 = (iz > 0) && (MB(m, X3MAX) > ms->x3max - 0.5*lz);
    if (shear_x1 && (lo1 || hi1)) {
      /* a radial face: wrap x, shift y by the (folded) shear offset, wrap y and z, route to the
       * face block on the other side at the new (y, z); the registers move with the position */
      const int cross_in = lo1;
      const double lxm = ms->x1max - ms->x1min;
      PR(DUSTB_IPX, p) += cross_in ? lxm : -lxm;
      PR(DUSTB_IPX1, p) += cross_in ? lxm : -lxm;
      const double lym = ms->x2max - ms->x2min;
      double ynew = PR(DUSTB_IPY, p) + (cross_in ? -ysh : ysh);
      if (ynew < ms->x2min) ynew += lym;
      if (ynew >= ms->x2max) ynew -= lym;
      const double dy = ynew - PR(DUSTB_IPY, p);
      PR(DUSTB_IPY, p) = ynew;
      PR(DUSTB_IPY1, p) += dy;
      const double lzm = ms->x3max - ms->x3min;
      if (lo3) { PR(DUSTB_IPZ, p) += lzm; PR(DUSTB_IPZ1, p) += lzm; }
      else if (hi3) { PR(DUSTB_IPZ, p) -= lzm; PR(DUSTB_IPZ1, p) -= lzm; }
      int b2 = (int)(((PR(DUSTB_IPY, p) - ms->x2min)/lym)*(double)ms->sb_nb2);
      b2 = (b2 < 0) ? 0 : ((b2 > ms->sb_nb2 - 1) ? ms->sb_nb2 - 1 : b2);
      int b3 = (int)(((PR(DUSTB_IPZ, p) - ms->x3min)/lzm)*(double)ms->sb_nb3);
      b3 = (b3 < 0) ? 0 : ((b3 > ms->sb_nb3 - 1) ? ms->sb_nb3 - 1 : b3);
      PI(DUSTB_PGID, p) = ms->sb_gid[((size_t)(cross_in ? 1 : 0)*ms->sb_nb3 + b3)*ms->sb_nb2 + b2];
      continue;
    }
    int gid = -1;
    if (!ms->nghbr_ml) gid = ms->nghbr[(size_t)m*27 + (iz + 1)*9 + (iy + 1)*3 + (ix + 1)];
    else if (ms->mb_lev) gid = 0;   /* refined mesh: found below from the new position */
    if (gid < 0) { err |= DUSTB_ERR_NGHBR; continue; }
    if (lo1) { PR(DUSTB_IPX, p) += ms->x1max - ms->x1min; PR(DUSTB_IPX1, p) += ms->x1max - ms->x1min; }
    else if (hi1) { PR(DUSTB_IPX, p) -= ms->x1max - ms->x1min; PR(DUSTB_IPX1, p) -= ms->x1max - ms->x1min; }
    if (lo2) { PR(DUSTB_IPY, p) += ms->x2max - ms->x2min; PR(DUSTB_IPY1, p) += ms->x2max - ms->x2min; }
    else if (hi2) { PR(DUSTB_IPY, p) -= ms->x2max - ms->x2min; PR(DUSTB_IPY1, p) -= ms->x2max - ms->x2min; }
    if (lo3) { PR(DUSTB_IPZ, p) += ms->x3max - ms->x3min; PR(DUSTB_IPZ1, p) += ms->x3max - ms->x3min; }
    else if (hi3) { PR(DUSTB_IPZ, p) -= ms->x3max - ms->x3min; PR(DUSTB_IPZ1, p) -= ms->x3max - ms->x3min; }
    if (ms->nghbr_ml) {
      /* a refined mesh: the reference searches the 56 neighbour slots of the block
       * (bvals_part.cpp:312-394); this restatement finds the block whose half-open box holds
       * the (wrapped) position instead, by a search over every block, which is where that slot
       * search must lead on a valid tree */
      const double q1 = PR(DUSTB_IPX, p), q2 = PR(DUSTB_IPY, p), q3 = PR(DUSTB_IPZ, p);
      gid = -1;
      for (int b = 0; b < ms->nmb; ++b)
        if (q1 >= MB(b, X1MIN) && q1 < MB(b, X1MAX) && q2 >= MB(b, X2MIN) && q2 < MB(b, X2MAX) &&
            q3 >= MB(b, X3MIN) && q3 < MB(b, X3MAX)) { gid = b + ms->gids; break; }
      if (gid < 0) { err |= DUSTB_ERR_NGHBR; continue; }
    }
    PI(DUSTB_PGID, p) = gid;
  }
  return err;
}

/* DepositDrag imex scatter, src/dust/dust_pm.cpp:197-277 */
unsigned oracle_deposit_qp(const dustb_ctx *c, double a_dt, double sh) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  memset(c->f.qdep, 0, field_size(ms, 5)*sizeof(double));
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  unsigned err = 0;
  const int clo = ms->three_d ? 0 : 1, chi = ms->three_d ? 2 : 1;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) reduction(| : err)
  for (int p = 0; p < c->part.npart; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    int ip, jp, kp; double wx[3], wy[3], wz[3];
    particle_weights(c, &d, m, PR(DUSTB_IPX, p), PR(DUSTB_IPY, p) + sh*PR(DUSTB_IPX, p),
                     PR(DUSTB_IPZ, p), &ip, &jp, &kp, wx, wy, wz);
    if (!halo_ok(ms, &d, ip, jp, kp)) { err |= DUSTB_ERR_HALO; continue; }
    double vol = cell_volume(ms, m);
    double cj = a_dt/(PR(DUSTB_IPTS, p) + a_dt);
    double muc = PR(DUSTB_IPM, p)*cj/vol;
    double vx = PR(DUSTB_IPVX, p), vy = PR(DUSTB_IPVY, p), vz = PR(DUSTB_IPVZ, p);
    for (int cc = clo; cc <= chi; ++cc)
      for (int b = 0; b < 3; ++b) {
        double wcb = wz[cc]*wy[b]*muc;
        if (wcb == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
          double w = wcb*wx[a];
          int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
          deposit_add(&A5(c->f.qdep, 5, d, m, 0, kk, jj, ii), w);
          deposit_add(&A5(c->f.qdep, 5, d, m, 1, kk, jj, ii), w*vx);
          deposit_add(&A5(c->f.qdep, 5, d, m, 2, kk, jj, ii), w*vy);
          deposit_add(&A5(c->f.qdep, 5, d, m, 3, kk, jj, ii), w*vz);
        }
      }
  }
  return err;
}

/* the 26 same-level directions in NeighborIndex(ox1,ox2,ox3,0,0) order
 * (src/mesh/nghbr_index.hpp:29-55), the order RecvAndSumDeposit sums the buffers in */
static const int kDirOrder[26][3] = {
  {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0},
  {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 1, 0},
  {0, 0, -1}, {0, 0, 1},
  {-1, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {1, 0, 1},
  {0, -1, -1}, {0, 1, -1}, {0, -1, 1}, {0, 1, 1},
  {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
  {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};

/* PackAndSendDeposit + RecvAndSumDeposit, same-level, one rank (src/bvals/bvals_dep.cpp:
 * 249-309 indices, :320-560 pack and sum): the sender's ghost strip in direction -ox is added
 * to the receiver's active strip on side ox, buffer by buffer in NeighborIndex order. */
/* ---- shear-periodic x1 faces (3-D shearing box) ------------------------------------------ */

/* faces of block m: bit 1 the inner x1 face, bit 2 the outer (bvals_part.cpp:260-261) */
static int sb_faces(const dustb_mesh *ms, int m) {
  const double lx = MB(m, X1MAX) - MB(m, X1MIN);
  int f = 0;
  if (MB(m, X1MIN) < ms->x1min + 0.5*lx) f |= 1;
  if (MB(m, X1MAX) > ms->x1max - 0.5*lx) f |= 2;
  return f;
}

/* the x2 and x3 block indices of block m, from its lower corner */
static void sb_b23(const dustb_mesh *ms, int m, int *b2, int *b3) {
  *b2 = (int)floor((MB(m, X2MIN) - ms->x2min)/((ms->x2max - ms->x2min)/ms->sb_nb2) + 0.5);
  *b3 = (int)floor((MB(m, X3MIN) - ms->x3min)/((ms->x3max - ms->x3min)/ms->sb_nb3) + 0.5);
}

/* local index of the face block (face f, b3, b2), or -1 */
static int sb_block(const dustb_mesh *ms, int f, int b3, int b2) {
  const int g = ms->sb_gid[((size_t)f*ms->sb_nb3 + b3)*ms->sb_nb2 + b2] - ms->gids;
  return (g >= 0 && g < ms->nmb) ? g : -1;
}

/* the active cell owning cell (k, j, i) of block m, in active-relative indices at most one
 * block beyond the block (the plain neighbour table); 0 if no block owns it */
static int owner_cell(const dustb_mesh *ms, int m, int *k, int *j, int *i, int *mo) {
  const int o1 = (*i < 0) ? -1 : ((*i >= ms->nx1) ? 1 : 0);
  const int o2 = (*j < 0) ? -1 : ((*j >= ms->nx2) ? 1 : 0);
  const int o3 = (*k < 0) ? -1 : ((*k >= ms->nx3) ? 1 : 0);
  if ((o1 | o2 | o3) == 0) { *mo = m; return 1; }
  const int gid = ms->nghbr[(size_t)m*27 + (o3 + 1)*9 + (o2 + 1)*3 + (o1 + 1)];
  if (gid < 0) return 0;
  *mo = gid - ms->gids;
  *i -= o1*ms->nx1; *j -= o2*ms->nx2; *k -= o3*ms->nx3;
  return 1;
}

/* PLM_RemapFlx and the update a - (flx(j+1) - flx(j)) of ShearingBoxCC::PackAndSend
 * (src/shearing_box/remap_fluxes.hpp:30-55, shearing_box_cc.cpp:118-140) at one row, from
 * g[t] = the row's column at rows r - 2 + t, t = 0..4 */
static double sb_remap(const double g[5], double eps) {
  double f[2];
  for (int h = 0; h < 2; ++h) {
    const int q = 2 + h;                 /* face between rows q-1 and q of g */
    double dql, dqr;
    if (eps > 0.0) { dql = g[q-1] - g[q-2]; dqr = g[q] - g[q-1]; }
    else { dql = g[q] - g[q-1]; dqr = g[q+1] - g[q]; }
    const double dq2 = dql*dqr;
    double dqm = 2.0*dq2/(dql + dqr);
    if (dq2 <= 0.0) dqm = 0.0;
    f[h] = (eps > 0.0) ? eps*(g[q-1] + 0.5*(1.0 - eps)*dqm) : eps*(g[q] - 0.5*(1.0 + eps)*dqm);
  }
  return g[2] - (f[1] - f[0]);
}

/* ShearingBoxCC::PackAndSend + RecvAndUnpack on one device (the conservative PLM remap of the
 * x1 ghost strips after the plain periodic copy, shearing_box_cc.cpp:78-197, integer pieces
 * shearing_box.cpp:260-330): the ghost strip of a face block at row J (its y-ghost rows and
 * x3 ghost planes included) takes the remapped periodic strip of the face block holding row
 * J - joffset (inner face; + joffset at the outer), joffset + eps = q Omega Lx t / dy.  The
 * periodic strip is read from the active cells that the plain copy takes it from. */
static void shear_copy(const dustb_ctx *c, double *a, int nvar) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  if (!ms->shear_x1 || !ms->three_d) return;
  const double lx = ms->x1max - ms->x1min;
  const double yshear = (c->phys.qshear*c->phys.omega0)*lx*ms->time;
  const int nb2 = ms->sb_nb2, nb3 = ms->sb_nb3;
  const long long Ny = (long long)nb2*ms->nx2;
  for (int n = 0; n < 2; ++n)
    for (int b3 = 0; b3 < nb3; ++b3)
      for (int b2 = 0; b2 < nb2; ++b2) {
        const int T = sb_block(ms, n, b3, b2);
        if (T < 0) continue;
        const double dy = MB(T, DX2);
        const long long joffset = (long long)(yshear/dy);
        double eps = fmod(yshear, dy)/dy;
        if (n == 1) eps *= -1.0;
        for (int v = 0; v < nvar; ++v)
          for (int k = 0; k < d.n3; ++k)
            for (int j = 0; j < d.n2; ++j)
              for (int i = 0; i < ms->ng; ++i) {
                const long long J = (long long)b2*ms->nx2 + (j - d.js);
                long long R = (n == 0) ? J - joffset : J + joffset;
                R %= Ny; if (R < 0) R += Ny;
                const int S = sb_block(ms, n, b3, (int)(R/ms->nx2));
                if (S < 0) continue;
                const int r = (int)(R % ms->nx2);          /* active-relative row of S */
                const int xr = (n == 0) ? i - ms->ng : ms->nx1 + i;
                double g[5];
                int ok = 1;
                for (int t = 0; t < 5 && ok; ++t) {
                  int kk = k - d.ks, jj = r - 2 + t, ii = xr, mo;
                  ok = owner_cell(ms, S, &kk, &jj, &ii, &mo);
                  if (ok) g[t] = A5(a, nvar, d, mo, v, d.ks + kk, d.js + jj, d.is + ii);
                }
                if (!ok) continue;
                A5(a, nvar, d, T, v, k, j, (n == 0) ? i : d.ie + 1 + i) = sb_remap(g, eps);
              }
      }
}

/* whether direction o1 from block m crosses a shear-periodic x1 face (those ghost cells are
 * remapped, not exchanged plainly) */
static int shear_crossing(const dustb_ctx *c, int m, int o1) {
  const dustb_mesh *ms = &c->mesh;
  if (!ms->shear_x1 || !ms->three_d || o1 == 0) return 0;
  const int f = sb_faces(ms, m);
  return (o1 < 0) ? (f & 1) : ((f & 2) != 0);
}

/* The shear part of the deposit remap (DepRemapPlan part 1, bvals_dep_general.cpp:99-240) for
 * active cell (k, j, i) of face block m: the ghost cells beyond the opposite x1 face, moved by
 * the box length and shifted in x2 by +shR (beyond the outer face) or -shR (beyond the inner
 * face) cells, add w * value, w = their overlap with the cell (piecewise-constant remap).
 * Source ghost planes in x3 reach the cell through the periodic wrap or, at a physical face,
 * the fold.  Sources in a fixed order: faces (inner-face targets first), source planes (the
 * cell's plane, then the ghost plane below or folded, then above), source blocks along x2
 * (offsets -1, 0, 1, each block once), source rows, images. */
static double shear_remap_entries(const dustb_ctx *c, const Ind *d, const double *a, int nvar,
                                  int m, int v, int k, int j, int i, double *scat,
                                  double tval);
static double shear_add_sum(const dustb_ctx *c, const Ind *d, const double *a, int nvar,
                            int m, int v, int k, int j, int i) {
  return shear_remap_entries(c, d, a, nvar, m, v, k, j, i, NULL, 0.0);
}
/* The entries of the cell's remap: with scat == NULL the sum of w * source value, else the
 * transpose, w * tval added into each source cell of scat (a field of the same shape). */
static double shear_remap_entries(const dustb_ctx *c, const Ind *d, const double *a, int nvar,
                                  int m, int v, int k, int j, int i, double *scat,
                                  double tval) {
  const dustb_mesh *ms = &c->mesh;
  const int faces = sb_faces(ms, m);
  const int ng1 = ms->ng - 1;
  const double lx = ms->x1max - ms->x1min, ly = ms->x2max - ms->x2min;
  const double ysh = fmod(c->phys.qshear*c->phys.omega0*lx*ms->time, ly);
  const long long N2 = (long long)ms->sb_nb2*ms->nx2;
  const double shR = ysh*(double)N2/ly;
  int b2, b3;
  sb_b23(ms, m, &b2, &b3);
  const int nb2 = ms->sb_nb2, nb3 = ms->sb_nb3;
  const long long J = (long long)b2*ms->nx2 + (j - d->js);
  double sum = 0.0;
  for (int side = 0; side < 2; ++side) {
    /* side 0: this block at the inner face, sources beyond the outer face (+shR) */
    if (!(faces & (side ? 2 : 1))) continue;
    const int g = side ? i - (d->ie - ng1) : i - d->is;
    if (g < 0 || g > ng1) continue;
    const int sface = side ? 0 : 1;
    const int si = side ? g : d->ie + 1 + g;                 /* source ghost column */
    const double sh = side ? -shR : shR;
    const long long F = (long long)floor((double)J - sh);
    for (int zc = 0; zc < 3; ++zc) {
      int sb3 = b3, sk = k;
      if (zc == 1) {                                        /* below the cell's plane */
        if (k > d->ks + ng1) continue;
        if (b3 > 0 || ms->x3bc == 0) { sb3 = (b3 + nb3 - 1) % nb3; sk = k + ms->nx3; }
        else if (!c->phys.x3_deposit_drop) { sk = 2*d->ks - 1 - k; }
        else continue;
      } else if (zc == 2) {                                 /* above */
        if (k < d->ke - ng1) continue;
        if (b3 < nb3 - 1 || ms->x3bc == 0) { sb3 = (b3 + 1) % nb3; sk = k - ms->nx3; }
        else if (!c->phys.x3_deposit_drop) { sk = 2*d->ke + 1 - k; }
        else continue;
      }
      const long long Fm = ((F % N2) + N2) % N2;
      const int bc = (int)(Fm/ms->nx2);
      int seen[3] = {-1, -1, -1};
      for (int db = -1; db <= 1; ++db) {
        const int sb2 = ((bc + db) % nb2 + nb2) % nb2;
        if (sb2 == seen[0] || sb2 == seen[1]) continue;
        seen[db + 1] = sb2;
        const int S = sb_block(ms, sface, sb3, sb2);
        if (S < 0) continue;
        for (long long Yc = F - 1; Yc <= F + 1; ++Yc)
          for (int q = -2; q <= 2; ++q) {
            /* the source row Yc + q N2 of S's strip (its ghost rows included) */
            const long long Y = Yc + q*N2;
            const long long sj = Y - (long long)sb2*ms->nx2 + d->js;
            if (sj < 0 || sj >= d->n2) continue;
            const double ya = (double)Y + sh, yb = (double)(Y + 1) + sh;
            for (int im = -2; im <= 2; ++im) {
              const double clo = (double)(J + im*N2), chi = clo + 1.0;
              const double o = fmin(yb, chi) - fmax(ya, clo);
              if (!(o > 0.0)) continue;
              if (scat) A5(scat, nvar, (*d), S, v, sk, (int)sj, si) += o*tval;
              else sum += o*A5(a, nvar, (*d), S, v, sk, (int)sj, si);
            }
          }
      }
    }
  }
  return sum;
}

void oracle_ghost_add(const dustb_ctx *c, double *a, int nvar) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  const int ng1 = ms->ng - 1;
  const int ndir = ms->three_d ? 26 : (ms->multi_d ? 8 : 2);
  /* pack every buffer first (the sends complete before any receive sums) */
  size_t total = 0;
  int lo[26][3], hi[26][3];
  for (int n = 0; n < ndir; ++n) {
    const int *o = kDirOrder[n];
    int s[3] = {d.is, d.js, d.ks}, e[3] = {d.ie, d.je, d.ke};
    for (int ax = 0; ax < 3; ++ax) {
      lo[n][ax] = (o[ax] > 0) ? (e[ax] - ng1) : s[ax];
      hi[n][ax] = (o[ax] < 0) ? (s[ax] + ng1) : e[ax];
    }
    total += (size_t)(hi[n][0] - lo[n][0] + 1)*(hi[n][1] - lo[n][1] + 1)*(hi[n][2] - lo[n][2] + 1);
  }
  double *buf = (double *)malloc(total*(size_t)ms->nmb*nvar*sizeof(double));
  size_t off = 0;
  size_t boff[26];
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  for (int n = 0; n < ndir; ++n) {
    boff[n] = off;
    size_t cnt = (size_t)(hi[n][0] - lo[n][0] + 1)*(hi[n][1] - lo[n][1] + 1)*(hi[n][2] - lo[n][2] + 1);
    off += cnt*(size_t)ms->nmb*nvar;
  }
  /* receiver m, buffer n (neighbour in direction o): values of the neighbour's ghost cells
   * at receiver index - o*nx */
  for (int m = 0; m < ms->nmb; ++m)
    for (int n = 0; n < ndir; ++n) {
      const int *o = kDirOrder[n];
      int gid = ms->nghbr[(size_t)m*27 + (o[2] + 1)*9 + (o[1] + 1)*3 + (o[0] + 1)];
      if (gid < 0 || shear_crossing(c, m, o[0])) continue;
      int src = gid - ms->gids;
      size_t q = boff[n] + (size_t)m*nvar*((hi[n][0]-lo[n][0]+1)*(hi[n][1]-lo[n][1]+1)*(hi[n][2]-lo[n][2]+1));
      for (int v = 0; v < nvar; ++v)
        for (int k = lo[n][2]; k <= hi[n][2]; ++k)
          for (int j = lo[n][1]; j <= hi[n][1]; ++j)
            for (int i = lo[n][0]; i <= hi[n][0]; ++i)
              buf[q++] = A5(a, nvar, d, src, v, k - o[2]*nx[2], j - o[1]*nx[1], i - o[0]*nx[0]);
    }
  for (int m = 0; m < ms->nmb; ++m)
    for (int n = 0; n < ndir; ++n) {
      const int *o = kDirOrder[n];
      int gid = ms->nghbr[(size_t)m*27 + (o[2] + 1)*9 + (o[1] + 1)*3 + (o[0] + 1)];
      if (gid < 0 || shear_crossing(c, m, o[0])) continue;
      size_t q = boff[n] + (size_t)m*nvar*((hi[n][0]-lo[n][0]+1)*(hi[n][1]-lo[n][1]+1)*(hi[n][2]-lo[n][2]+1));
      for (int v = 0; v < nvar; ++v)
        for (int k = lo[n][2]; k <= hi[n][2]; ++k)
          for (int j = lo[n][1]; j <= hi[n][1]; ++j)
            for (int i = lo[n][0]; i <= hi[n][0]; ++i)
              A5(a, nvar, d, m, v, k, j, i) += buf[q++];
    }
  free(buf);
  /* physical x3 faces, fold mode (DepRemapPlan x3mode 1, src/bvals/bvals_dep_general.cpp:
   * 130-140: a ghost interval beyond the face is mirrored about it): the ghost plane ks-1-t
   * (ke+1+t) is added into the active plane ks+t (ke-t), the block's own column first, then
   * the x1/x2 neighbours' ghost strips facing the cell, in NeighborIndex order.  (The
   * reference sums a target's contributions in (source gid, source cell) order; the sums here
   * differ from it by rounding only.)  The ghost cells read are untouched by the exchange. */
  if (ms->three_d && ms->x3bc != 0 && !c->phys.x3_deposit_drop)
  for (int m = 0; m < ms->nmb; ++m)
    for (int side = 0; side < 2; ++side) {
      const int o3 = side ? 1 : -1;
      if (ms->nghbr[(size_t)m*27 + (o3 + 1)*9 + 1*3 + 1] >= 0) continue;
      for (int t = 0; t < ms->ng; ++t) {
        const int k = side ? d.ke - t : d.ks + t;
        const int kg = side ? d.ke + 1 + t : d.ks - 1 - t;
        for (int v = 0; v < nvar; ++v)
          for (int j = d.js; j <= d.je; ++j)
            for (int i = d.is; i <= d.ie; ++i) {
              double val = A5(a, nvar, d, m, v, k, j, i) + A5(a, nvar, d, m, v, kg, j, i);
              for (int n = 0; n < ndir; ++n) {
                const int *o = kDirOrder[n];
                if (o[2] != 0) continue;
                if (o[0] > 0 && i < d.ie - ng1) continue;
                if (o[0] < 0 && i > d.is + ng1) continue;
                if (o[1] > 0 && j < d.je - ng1) continue;
                if (o[1] < 0 && j > d.js + ng1) continue;
                int gid = ms->nghbr[(size_t)m*27 + 1*9 + (o[1] + 1)*3 + (o[0] + 1)];
                if (gid < 0 || shear_crossing(c, m, o[0])) continue;
                val += A5(a, nvar, d, gid - ms->gids, v, kg, j - o[1]*nx[1], i - o[0]*nx[0]);
              }
              A5(a, nvar, d, m, v, k, j, i) = val;
            }
      }
    }
  /* shear-periodic x1 faces: the ghost cells beyond them, remapped (the sums of the sources
   * are added to the cells as DepRemapPlan adds them, GeneralApply) */
  if (!ms->shear_x1 || !ms->three_d) return;
  const size_t ncell = (size_t)d.n1*d.n2*d.n3;
  double *add = (double *)calloc((size_t)ms->nmb*nvar*ncell, sizeof(double));
  for (int m = 0; m < ms->nmb; ++m) {
    if (!sb_faces(ms, m)) continue;
    for (int v = 0; v < nvar; ++v)
      for (int k = d.ks; k <= d.ke; ++k)
        for (int j = d.js; j <= d.je; ++j)
          for (int i = d.is; i <= d.ie; ++i)
            add[(((size_t)m*nvar + v)*d.n3 + k)*d.n2*d.n1 + (size_t)j*d.n1 + i] =
                shear_add_sum(c, &d, a, nvar, m, v, k, j, i);
  }
  /* (all sums read the ghost cells before any cell changes: they are never written) */
  for (int m = 0; m < ms->nmb; ++m) {
    if (!sb_faces(ms, m)) continue;
    for (int v = 0; v < nvar; ++v)
      for (int k = d.ks; k <= d.ke; ++k)
        for (int j = d.js; j <= d.je; ++j)
          for (int i = d.is; i <= d.ie; ++i)
            A5(a, nvar, d, m, v, k, j, i) += add[(((size_t)m*nvar + v)*d.n3 + k)*d.n2*d.n1 + (size_t)j*d.n1 + i];
  }
  free(add);
}


/* UstarX3BCs, src/dust/dust_tasks.cpp:445-469 (single level) */
static void ustar_x3_bcs(const dustb_ctx *c, double *a) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  if (!ms->three_d || ms->x3bc == 0) return;
  const int refl = (ms->x3bc == 1);
  for (int m = 0; m < ms->nmb; ++m) {
    int lo_face = ms->nghbr[(size_t)m*27 + 0*9 + 1*3 + 1] < 0;
    int hi_face = ms->nghbr[(size_t)m*27 + 2*9 + 1*3 + 1] < 0;
    for (int g = 0; g < ms->ng; ++g)
      for (int j = 0; j < d.n2; ++j)
        for (int i = 0; i < d.n1; ++i) {
          if (lo_face) {
            int kg = d.ks - 1 - g, kc = refl ? (d.ks + g) : d.ks;
            for (int v = 0; v < 3; ++v)
              A5(a, 3, d, m, v, kg, j, i) = (refl && v == 2) ? -A5(a, 3, d, m, v, kc, j, i)
                                                             : A5(a, 3, d, m, v, kc, j, i);
          }
          if (hi_face) {
            int kg = d.ke + 1 + g, kc = refl ? (d.ke - g) : d.ke;
            for (int v = 0; v < 3; ++v)
              A5(a, 3, d, m, v, kg, j, i) = (refl && v == 2) ? -A5(a, 3, d, m, v, kc, j, i)
                                                             : A5(a, 3, d, m, v, kc, j, i);
          }
        }
  }
}

/* MeshBoundaryValuesCC same-level copy exchange: every ghost cell takes the neighbour's
 * active cell at index - o*nx (InitSendIndices/InitRecvIndices of the CC exchange), then
 * the x3 physical boundary values when x3_bcs */
void oracle_ghost_copy(const dustb_ctx *c, double *a, int nvar, int x3_bcs) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = 0; k < d.n3; ++k)
      for (int j = 0; j < d.n2; ++j)
        for (int i = 0; i < d.n1; ++i) {
          int o[3];
          o[0] = (i < d.is) ? -1 : ((i > d.ie) ? 1 : 0);
          o[1] = (j < d.js) ? -1 : ((j > d.je) ? 1 : 0);
          o[2] = (k < d.ks) ? -1 : ((k > d.ke) ? 1 : 0);
          if (o[0] == 0 && o[1] == 0 && o[2] == 0) continue;
          int gid = ms->nghbr[(size_t)m*27 + (o[2] + 1)*9 + (o[1] + 1)*3 + (o[0] + 1)];
          if (gid < 0) continue;
          int src = gid - ms->gids;
          for (int v = 0; v < nvar; ++v)
            A5(a, nvar, d, m, v, k, j, i) =
                A5(a, nvar, d, src, v, k - o[2]*nx[2], j - o[1]*nx[1], i - o[0]*nx[0]);
        }
  shear_copy(c, a, nvar);
  if (x3_bcs && nvar == 3) ustar_x3_bcs(c, a);
}

/* dust_ustar (dust_pm.cpp:426-436) == dust_solver_local_guess (dust_solver.cpp:643-649) */
void oracle_solve_ustar(const dustb_ctx *c) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  const int br = c->phys.back_reaction;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i) {
          double q0 = br ? A5(c->f.qdep, 5, d, m, 0, k, j, i) : 0.0;
          double denom = 1.0/(A5(c->f.u0, nv, d, m, 0, k, j, i) + q0);
          for (int v = 0; v < 3; ++v) {
            double qv = br ? A5(c->f.qdep, 5, d, m, 1 + v, k, j, i) : 0.0;
            A5(c->f.ustar, 3, d, m, v, k, j, i) = (A5(c->f.u0, nv, d, m, 1 + v, k, j, i) + qv)*denom;
          }
        }
}

/* PointOperatorParticles, src/dust/dust_solver.cpp:126-203 */
static unsigned operator_particles(const dustb_ctx *c, const double *field, double *result,
                                   double a_dt, double sh) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int clo = ms->three_d ? 0 : 1, chi = ms->three_d ? 2 : 1;
  unsigned err = 0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) reduction(| : err)
  for (int p = 0; p < c->part.npart; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    int ip, jp, kp; double wx[3], wy[3], wz[3];
    particle_weights(c, &d, m, PR(DUSTB_IPX, p), PR(DUSTB_IPY, p) + sh*PR(DUSTB_IPX, p),
                     PR(DUSTB_IPZ, p), &ip, &jp, &kp, wx, wy, wz);
    if (!halo_ok(ms, &d, ip, jp, kp)) { err |= DUSTB_ERR_HALO; continue; }
    double g[3] = {0.0, 0.0, 0.0};
    for (int cc = clo; cc <= chi; ++cc)
      for (int b = 0; b < 3; ++b) {
        double wcb = wz[cc]*wy[b];
        if (wcb == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
          double w = wcb*wx[a];
          int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
          g[0] += w*A5(field, 3, d, m, 0, kk, jj, ii);
          g[1] += w*A5(field, 3, d, m, 1, kk, jj, ii);
          g[2] += w*A5(field, 3, d, m, 2, kk, jj, ii);
        }
      }
    double vol = cell_volume(ms, m);
    double cj = a_dt/(PR(DUSTB_IPTS, p) + a_dt);
    double fac = PR(DUSTB_IPM, p)*cj/vol;
    for (int cc = clo; cc <= chi; ++cc)
      for (int b = 0; b < 3; ++b) {
        double wcb = wz[cc]*wy[b]*fac;
        if (wcb == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
          double w = wcb*wx[a];
          int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
          deposit_add(&A5(result, 3, d, m, 0, kk, jj, ii), w*g[0]);
          deposit_add(&A5(result, 3, d, m, 1, kk, jj, ii), w*g[1]);
          deposit_add(&A5(result, 3, d, m, 2, kk, jj, ii), w*g[2]);
        }
      }
  }
  return err;
}

/* the per-cell correction of ApplyCoupledOperatorImpl (dust_solver.cpp:240-252):
 * u* += (rho + Q)^-1 (rho u + P - rho u* - result), result = work */
void oracle_dc_correct(const dustb_ctx *c) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  double *x = c->f.ustar, *r = c->f.work;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i) {
          double rho = A5(c->f.u0, nv, d, m, 0, k, j, i);
          double pinv = 1.0/(rho + A5(c->f.qdep, 5, d, m, 0, k, j, i));
          for (int v = 0; v < 3; ++v) {
            double av = A5(r, 3, d, m, v, k, j, i) + rho*A5(x, 3, d, m, v, k, j, i);
            double rv = A5(c->f.u0, nv, d, m, 1 + v, k, j, i) +
                        A5(c->f.qdep, 5, d, m, 1 + v, k, j, i) - av;
            A5(x, 3, d, m, v, k, j, i) += pinv*rv;
          }
        }
}

/* PointOperatorParticles of u* into work (work not cleared; sh = 0) */
unsigned oracle_operator_particles(const dustb_ctx *c, double a_dt) {
  return operator_particles(c, c->f.ustar, c->f.work, a_dt, 0.0);
}

/* ApplyDefectCorrection -> ApplyCoupledOperatorImpl(correct_field = true),
 * src/dust/dust_solver.cpp:218-252 */
unsigned oracle_dc1_sweep(const dustb_ctx *c, double a_dt, double sh) {
  const dustb_mesh *ms = &c->mesh;
  double *x = c->f.ustar, *r = c->f.work;
  oracle_ghost_copy(c, x, 3, 1);
  memset(r, 0, field_size(ms, 3)*sizeof(double));
  unsigned err = operator_particles(c, x, r, a_dt, sh);
  oracle_ghost_add(c, r, 3);
  oracle_dc_correct(c);
  return err;
}

/* GatherKickPMBR point particles, src/dust/dust_pm.cpp:450-568 */
unsigned oracle_gather_kick_pmbr(const dustb_ctx *c, double a_dt, double sh) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  const int br = c->phys.back_reaction;
  if (br) memset(c->f.dmom, 0, field_size(ms, 3)*sizeof(double));
  double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int clo = ms->three_d ? 0 : 1, chi = ms->three_d ? 2 : 1;
  unsigned err = 0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) reduction(| : err)
  for (int p = 0; p < c->part.npart; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    int ip, jp, kp; double wx[3], wy[3], wz[3];
    particle_weights(c, &d, m, PR(DUSTB_IPX, p), PR(DUSTB_IPY, p) + sh*PR(DUSTB_IPX, p),
                     PR(DUSTB_IPZ, p), &ip, &jp, &kp, wx, wy, wz);
    if (!halo_ok(ms, &d, ip, jp, kp)) { err |= DUSTB_ERR_HALO; continue; }
    double ux = 0.0, uy = 0.0, uz = 0.0;
    for (int cc = clo; cc <= chi; ++cc)
      for (int b = 0; b < 3; ++b) {
        double wcb = wz[cc]*wy[b];
        if (wcb == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
          double w = wcb*wx[a];
          int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
          ux += w*A5(c->f.ustar, 3, d, m, 0, kk, jj, ii);
          uy += w*A5(c->f.ustar, 3, d, m, 1, kk, jj, ii);
          uz += w*A5(c->f.ustar, 3, d, m, 2, kk, jj, ii);
        }
      }
    double cj = a_dt/(PR(DUSTB_IPTS, p) + a_dt);
    double dvx = cj*(ux - PR(DUSTB_IPVX, p));
    double dvy = cj*(uy - PR(DUSTB_IPVY, p));
    double dvz = cj*(uz - PR(DUSTB_IPVZ, p));
    PR(DUSTB_IPVX, p) += dvx; PR(DUSTB_IPVY, p) += dvy; PR(DUSTB_IPVZ, p) += dvz;
    PR(DUSTB_IPRX, p) = dvx/a_dt; PR(DUSTB_IPRY, p) = dvy/a_dt; PR(DUSTB_IPRZ, p) = dvz/a_dt;
    if (br) {
      double vol = cell_volume(ms, m);
      double fac = -PR(DUSTB_IPM, p)/vol;
      for (int cc = clo; cc <= chi; ++cc)
        for (int b = 0; b < 3; ++b) {
          double wcb = wz[cc]*wy[b]*fac;
          if (wcb == 0.0) continue;
          for (int a = 0; a < 3; ++a) {
            double w = wcb*wx[a];
            int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
            deposit_add(&A5(c->f.dmom, 3, d, m, 0, kk, jj, ii), w*dvx);
            deposit_add(&A5(c->f.dmom, 3, d, m, 1, kk, jj, ii), w*dvy);
            deposit_add(&A5(c->f.dmom, 3, d, m, 2, kk, jj, ii), w*dvz);
          }
        }
    }
  }
  return err;
}

/* ApplyPMBR imex, src/dust/dust_pm.cpp:605-711 (consistent point split :624-697) */
void oracle_apply_pmbr(const dustb_ctx *c, double a_dt) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  if (!c->phys.back_reaction) return;
  const double inv_adt = 1.0/a_dt;
  double *u0 = c->f.u0, *dm = c->f.dmom;
  if (!c->phys.consistent_gas) {
    for (int m = 0; m < ms->nmb; ++m)
      for (int k = d.ks; k <= d.ke; ++k)
        for (int j = d.js; j <= d.je; ++j)
          for (int i = d.is; i <= d.ie; ++i)
            for (int v = 0; v < 3; ++v) {
              A5(u0, nv, d, m, 1 + v, k, j, i) += A5(dm, 3, d, m, v, k, j, i);
              A5(dm, 3, d, m, v, k, j, i) *= inv_adt;
            }
    return;
  }
  double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  double *res = c->f.resid;
  memset(res, 0, field_size(ms, 4)*sizeof(double));
  for (int p = 0; p < c->part.npart; ++p) {     /* dust_imex_point_center_mass */
    if (PR(DUSTB_IPM, p) <= 0.0) continue;
    int m = PI(DUSTB_PGID, p) - ms->gids;
    int ip, jp, kp; double w[3];
    pm_weights(PR(DUSTB_IPX, p), MB(m, X1MIN), MB(m, X1MAX), ms->nx1, d.is, c->phys.scheme, &ip, w);
    pm_weights(PR(DUSTB_IPY, p), MB(m, X2MIN), MB(m, X2MAX), ms->nx2, d.js, c->phys.scheme, &jp, w);
    if (ms->three_d) pm_weights(PR(DUSTB_IPZ, p), MB(m, X3MIN), MB(m, X3MAX), ms->nx3, d.ks,
                                c->phys.scheme, &kp, w);
    else kp = d.ks;
    double vol = cell_volume(ms, m);
    deposit_add(&A5(res, 4, d, m, 3, kp, jp, ip),
                PR(DUSTB_IPM, p)*(a_dt/(PR(DUSTB_IPTS, p) + a_dt))/vol);
  }
  for (int m = 0; m < ms->nmb; ++m)              /* dust_imex_point_consistent_gas */
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i) {
          const double rho = A5(u0, nv, d, m, 0, k, j, i), qt = A5(res, 4, d, m, 3, k, j, i);
          const double q = A5(c->f.qdep, 5, d, m, 0, k, j, i);
          for (int v = 0; v < 3; ++v) {
            double dgas = A5(dm, 3, d, m, v, k, j, i);
            if (qt > 0.0) {
              const double g = rho*A5(c->f.ustar, 3, d, m, v, k, j, i) - A5(u0, nv, d, m, 1 + v, k, j, i);
              const double r = (A5(dm, 3, d, m, v, k, j, i) - g)/(rho + q);
              dgas = g + rho*r;
              A5(res, 4, d, m, v, k, j, i) = r*q/qt;
            }
            A5(u0, nv, d, m, 1 + v, k, j, i) += dgas;
            A5(dm, 3, d, m, v, k, j, i) = dgas*inv_adt;
          }
        }
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads)
  for (int p = 0; p < c->part.npart; ++p) {     /* dust_imex_point_consistent_dust */
    if (PR(DUSTB_IPM, p) <= 0.0) continue;
    int m = PI(DUSTB_PGID, p) - ms->gids;
    int ip, jp, kp; double w[3];
    pm_weights(PR(DUSTB_IPX, p), MB(m, X1MIN), MB(m, X1MAX), ms->nx1, d.is, c->phys.scheme, &ip, w);
    pm_weights(PR(DUSTB_IPY, p), MB(m, X2MIN), MB(m, X2MAX), ms->nx2, d.js, c->phys.scheme, &jp, w);
    if (ms->three_d) pm_weights(PR(DUSTB_IPZ, p), MB(m, X3MIN), MB(m, X3MAX), ms->nx3, d.ks,
                                c->phys.scheme, &kp, w);
    else kp = d.ks;
    const double cj = a_dt/(PR(DUSTB_IPTS, p) + a_dt);
    for (int v = 0; v < 3; ++v) {
      const double dv = cj*A5(res, 4, d, m, v, kp, jp, ip);
      PR(DUSTB_IPVX + 2*v, p) += dv;
      PR(DUSTB_IPRX + v, p) += dv/a_dt;
    }
  }
}

/* NewTimeStep, src/dust/dust_newdt.cpp:108-149 (the particle part, before the CFL factor) */
double oracle_newdt(const dustb_ctx *c) {
  const dustb_mesh *ms = &c->mesh;
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int shear3d = c->phys.shearing_box && ms->three_d;
  const double qo = c->phys.qshear*c->phys.omega0;
  double dtp = (double)FLT_MAX;
  for (int p = 0; p < c->part.npart; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    double vy = PR(DUSTB_IPVY, p);
    if (shear3d) vy -= qo*PR(DUSTB_IPX, p);
    dtp = fmin(MB(m, DX1)/fmax(fabs(PR(DUSTB_IPVX, p)), 1.0e-30), dtp);
    dtp = fmin(MB(m, DX2)/fmax(fabs(vy), 1.0e-30), dtp);
    if (ms->three_d) dtp = fmin(MB(m, DX3)/fmax(fabs(PR(DUSTB_IPVZ, p)), 1.0e-30), dtp);
  }
  return dtp;
}

/* RefreshStoppingTimeMaximum (validation + extrema), src/dust/dust_newdt.cpp:34-98 */
void oracle_tstop_extrema(const dustb_ctx *c, int nspecies, double out[2]) {
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  double mx = 0.0, mn = DBL_MAX;
  for (int p = 0; p < c->part.npart; ++p) {
    int s = PI(DUSTB_PSP, p);
    double ts = PR(DUSTB_IPTS, p);
    int bad = (s < 0 || (nspecies > 0 && s >= nspecies) || !isfinite(ts) || !(ts > 0.0));
    mx = fmax(mx, bad ? DBL_MAX : ts);
    mn = fmin(mn, ts);
  }
  out[0] = mx; out[1] = mn;
}

/* ---- SortParticles, src/dust/dust_cloud_device.cpp:1881-1977 ---------------------------- */
static int cmp_i64(const void *a, const void *b) {
  int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
  return (x > y) - (x < y);
}

/* the sort keys (block, k, j, i) of the floor() cell formula and the resulting permutation
 * (order[k] = old index of the particle that goes to slot k) */
void oracle_sort_order(const dustb_ctx *c, int *order, int64_t *cellkey) {
  const dustb_mesh *ms = &c->mesh;
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int n = c->part.npart;
  const int nx1 = ms->nx1, nx2 = ms->nx2, nx3 = ms->three_d ? ms->nx3 : 1;
  const int64_t ncell = (int64_t)nx1*nx2*nx3, np = n;
  int64_t *key = (int64_t *)malloc(sizeof(int64_t)*(size_t)(n > 0 ? n : 1));
  for (int p = 0; p < n; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    m = (m < 0) ? 0 : ((m >= ms->nmb) ? ms->nmb - 1 : m);
    int i = (int)floor((PR(DUSTB_IPX, p) - MB(m, X1MIN))/MB(m, DX1));
    int j = (int)floor((PR(DUSTB_IPY, p) - MB(m, X2MIN))/MB(m, DX2));
    i = (i < 0) ? 0 : ((i >= nx1) ? nx1 - 1 : i);
    j = (j < 0) ? 0 : ((j >= nx2) ? nx2 - 1 : j);
    int k = 0;
    if (ms->three_d) {
      k = (int)floor((PR(DUSTB_IPZ, p) - MB(m, X3MIN))/MB(m, DX3));
      k = (k < 0) ? 0 : ((k >= nx3) ? nx3 - 1 : k);
    }
    int64_t cell = ((int64_t)k*nx2 + j)*nx1 + i;
    key[p] = (m*ncell + cell)*np + p;
    if (cellkey) cellkey[p] = m*ncell + cell;
  }
  qsort(key, (size_t)n, sizeof(int64_t), cmp_i64);
  for (int k = 0; k < n; ++k) order[k] = (int)(key[k] % np);
  free(key);
}

void oracle_sort_particles(const dustb_ctx *c, double *spare_pr, int *spare_pi) {
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int n = c->part.npart;
  int *order = (int *)malloc(sizeof(int)*(size_t)(n > 0 ? n : 1));
  oracle_sort_order(c, order, NULL);
  for (int k = 0; k < n; ++k) {
    int p = order[k];
    for (int r = 0; r < DUSTB_NREAL; ++r) spare_pr[(size_t)r*stride + k] = PR(r, p);
    for (int r = 0; r < DUSTB_NINT; ++r) spare_pi[(size_t)r*stride + k] = PI(r, p);
  }
  free(order);
}

void oracle_imex2p_coeffs(double gamma, double gam0[3], double gam1[3], double beta[3],
                          double *atw22);

/* ---- refinable clouds on a uniform mesh: plain P1 hat clouds ------------------------
 * CloudShape1D (src/dust/dust.hpp:240-298) with HatCDF / HatMoment (:169-182) for a cloud
 * without lobes: along each direction the hat of half-width ell = dx / 2^level about the
 * particle; a cell's weight is the difference of the hat CDF at its two faces, its first
 * moment about the particle ell times the difference of the moment antiderivative.
 * LeafTraversal3D::ForEach (src/dust/dust_leaf3d.hpp:368-513) on a uniform mesh: the cells of
 * the block and of its same-level neighbours that the support overlaps, each cell's faces
 * from its own block's origin (the neighbour's periodic image next to the block), weight w =
 * w1 w2 w3 and moments (g1 w2 w3, w1 g2 w3, w1 w2 g3); across a physical x3 face a second
 * part, the cloud mirrored about the face, its x3 moments taken about the particle (zcorr).
 * Leaf order here: part, z, y, x, each direction from the lower neighbour through the block to
 * the upper one; leaves of zero weight (and zero moments) are skipped.  2-D
 * (LeafTraversal::ForEach and LeafApi<LeafTraversal>, src/dust/dust_leaf_api.hpp:31-146): no x3
 * direction (a unit z axis: w = w2 w1 and the moments bit for bit), no orbital-advection
 * shift, the cell area as the measure, the coupled mass m (a_dt / (t_s + a_dt)). */
static double hat_cdf(double s) {
  if (s <= -1.0) return 0.0;
  if (s >= 1.0) return 1.0;
  return (s <= 0.0) ? 0.5*(1.0 + s)*(1.0 + s) : 1.0 - 0.5*(1.0 - s)*(1.0 - s);
}
static double hat_moment(double s) {
  if (s <= -1.0 || s >= 1.0) return 1.0/6.0;
  return (s <= 0.0) ? 0.5*(s*s) + (s*s)*s/3.0 : 0.5*(s*s) - (s*s)*s/3.0;
}

typedef struct { int n; int o[6]; int i[6]; double w[6]; double g[6]; double org[6]; } CloudAxis;

/* the cells of one direction a (0..2) for a cloud at x of level lev anchored at block m */
static void cloud_axis(const dustb_ctx *c, int m, int a, double x, int lev, CloudAxis *A) {
  const dustb_mesh *ms = &c->mesh;
  const int nx = (a == 0) ? ms->nx1 : ((a == 1) ? ms->nx2 : ms->nx3);
  const double L = (a == 0) ? ms->x1max - ms->x1min : ((a == 1) ? ms->x2max - ms->x2min
                                                                 : ms->x3max - ms->x3min);
  const double dx = MB(m, DX1 + a), idx = 1.0/dx;
  const double ell = ldexp(dx, -lev), inv = ldexp(idx, lev);
  const double lo = x - ell, hi = x + ell;
  A->n = 0;
  for (int o = -1; o <= 1; ++o) {
    int b = m;
    if (o != 0) {
      const int oo[3] = {a == 0 ? o : 0, a == 1 ? o : 0, a == 2 ? o : 0};
      const int gid = ms->nghbr[(size_t)m*27 + (oo[2] + 1)*9 + (oo[1] + 1)*3 + (oo[0] + 1)];
      if (gid < 0 || gid - ms->gids < 0 || gid - ms->gids >= ms->nmb) continue;
      b = gid - ms->gids;
    }
    double bx0 = MB(b, X1MIN + a);
    if (o < 0 && MB(b, X1MIN + a) >= MB(m, X1MIN + a)) bx0 -= L;   /* its image below m */
    if (o > 0 && MB(b, X1MIN + a) <= MB(m, X1MIN + a)) bx0 += L;   /* its image above m */
    int i0 = (int)floor((lo - bx0)*idx), i1 = (int)ceil((hi - bx0)*idx) - 1;
    i0 = (i0 < 0) ? 0 : i0;
    i1 = (i1 > nx - 1) ? nx - 1 : i1;
    for (int i = i0; i <= i1 && A->n < 6; ++i) {
      const double za = (bx0 + i*dx - x)*inv, zb = (bx0 + (i + 1)*dx - x)*inv;
      A->o[A->n] = o; A->i[A->n] = i; A->org[A->n] = bx0;
      A->w[A->n] = hat_cdf(zb) - hat_cdf(za);
      A->g[A->n] = ell*(hat_moment(zb) - hat_moment(za));
      ++A->n;
    }
  }
}

/* Frame: the periodic image of the position next to block m; then whether this restatement
 * takes the cloud: a level code without lobe bits and a position inside the block (slack: within
 * that many cells of it, the pc2 midpoint) */
static int cloud_frame_ok(const dustb_ctx *c, int m, double x[3], int code, double slack) {
  const dustb_mesh *ms = &c->mesh;
  const int bits = ms->leaf ? (15 | (3 << 4) | (3 << 6) | (3 << 9)) : 15;
  if (m < 0 || m >= ms->nmb || (code & ~bits) != 0) return 0;
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  const double L[3] = {ms->x1max - ms->x1min, ms->x2max - ms->x2min, ms->x3max - ms->x3min};
  for (int a = 0; a < (ms->three_d ? 3 : 2); ++a) {
    const double cx = MB(m, X1MIN + a) + 0.5*nx[a]*MB(m, DX1 + a);
    x[a] -= L[a]*round((x[a] - cx)*(1.0/L[a]));
    const double e = slack*MB(m, DX1 + a);
    if (!(x[a] >= MB(m, X1MIN + a) - e && x[a] < MB(m, X1MAX + a) + e)) return 0;
  }
  return 1;
}

/* the stage position (3-D: y + sh x; 2-D: no shift) */
static void cloud_position(const dustb_ctx *c, int p, double sh, double x[3]) {
  const double *pr = c->part.pr; long long stride = c->part.stride;
  if (c->mesh.three_d) {
    x[0] = PR(DUSTB_IPX, p); x[1] = PR(DUSTB_IPY, p) + sh*PR(DUSTB_IPX, p); x[2] = PR(DUSTB_IPZ, p);
  } else {
    x[0] = PR(DUSTB_IPX, p); x[1] = PR(DUSTB_IPY, p); x[2] = 0.0;
  }
}
static double cloud_measure(const dustb_ctx *c, int b) {
  const dustb_mesh *ms = &c->mesh;
  return ms->three_d ? MB(b, DX1)*MB(b, DX2)*MB(b, DX3) : MB(b, DX1)*MB(b, DX2);
}
/* the owner block of a leaf in direction (ox, oy, oz) of m */
static int cloud_owner(const dustb_ctx *c, int m, int ox, int oy, int oz) {
  if (!ox && !oy && !oz) return m;
  const int gid = c->mesh.nghbr[(size_t)m*27 + (oz + 1)*9 + (oy + 1)*3 + (ox + 1)];
  const int b = gid - c->mesh.gids;
  return (gid < 0 || b < 0 || b >= c->mesh.nmb) ? -1 : b;
}

typedef struct { int b, k, j, i; double w, m1x, m1y, m1z; } CloudLeaf;
typedef void (*CloudLeafFn)(void *ctx, const CloudLeaf *lf);

/* ---- refinable clouds on a refined 3-D mesh: the leaf traversal (test restatement) ------
 * LeafTraversal3D (src/dust/dust_leaf3d.hpp), one rank, no shear.  The cloud shape along one
 * direction (CloudShape1D, src/dust/dust.hpp:240-298): a hat of half-width ell = root_dx /
 * 2^level about the particle, or with a transition lobe on one side (2/3) S_ell(x - xp) + (1/3)
 * S_ell(x - xp -/+ ell), or with both lobes the parent hat of half-width 2 ell; the weight of a
 * cell is the integral between its faces, its moment about the particle the integral of (x -
 * xp) (zero along lobed directions for gathers: the point rule of GatherCode).  The cells are
 * those of every candidate block under the support: the anchor alone when the support lies
 * inside it (ForEach :409-423), else the anchor and its distinct neighbours when they cover it
 * (NeedGlobal :253-272: the safe ring, else the band scan Covered :198-238), else every block
 * and periodic image (ForCandidates :142-180) that meets it; cells in the order part,
 * candidate, runs of four in x, z, y, x (:426-500).  Leaf tables: oracle_leaf_tables. */
typedef struct { double x, ell, inv, sl, lo, hi; int lobe, both, point; } Shape1;
static Shape1 make_shape(double x, double ell_in, double inv_in, int lobe_in, int point) {
  Shape1 s;
  s.both = (lobe_in == 3);
  s.ell = s.both ? 2.0*ell_in : ell_in;
  s.lobe = s.both ? 0 : lobe_in;
  s.sl = (s.lobe == 1) ? -s.ell : s.ell;
  s.lo = (s.lobe == 1) ? x - 2.0*s.ell : x - s.ell;
  s.hi = (s.lobe == 2) ? x + 2.0*s.ell : x + s.ell;
  s.x = x;
  s.point = point;
  s.inv = s.both ? 0.5*inv_in : inv_in;
  return s;
}
typedef struct { double c, cl, h, hl; } Face1;
static Face1 face_at(const Shape1 *s, double z, int mom) {
  Face1 f = {0.0, 0.0, 0.0, 0.0};
  const double sz = (z - s->x)*s->inv;
  f.c = hat_cdf(sz);
  if (mom) f.h = hat_moment(sz);
  if (s->lobe) {
    const double tz = (z - s->x - s->sl)*s->inv;
    f.cl = hat_cdf(tz);
    if (mom) f.hl = hat_moment(tz);
  }
  return f;
}
static void cell_1d(const Shape1 *s, const Face1 *a, const Face1 *b, int mom, double *w,
                    double *g) {
  *w = b->c - a->c;
  *g = 0.0;
  if (mom) *g = (s->both && s->point) ? 0.0 : s->ell*(b->h - a->h);
  if (s->lobe) {
    const double wl = b->cl - a->cl;
    *w = (2.0/3.0)*(*w) + (1.0/3.0)*wl;
    if (mom) *g = s->point ? 0.0 : (2.0/3.0)*(*g) + (1.0/3.0)*(s->ell*(b->hl - a->hl) + s->sl*wl);
  }
}

/* a candidate: block b moved by -(sx, sy, sz) domain lengths */
typedef struct { int b, s[3]; } Cand;
typedef struct { Cand *v; int n, cap; } CandList;
static void cand_push(CandList *L, int b, int sx, int sy, int sz) {
  if (L->n == L->cap) {
    L->cap = L->cap ? 2*L->cap : 128;
    L->v = (Cand *)realloc(L->v, (size_t)L->cap*sizeof(Cand));
  }
  Cand c = {b, {sx, sy, sz}};
  L->v[L->n++] = c;
}
static int fdiv(int a, int n) { return (int)floor((double)a/(double)n); }
/* the candidates of ForCandidates: local (m, then its neighbours) or global (every block's
 * periodic images meeting the finest-cell box widened by r), appended to L */
static void candidates(const dustb_ctx *c, int m, int global, const int box[6], int r,
                       CandList *L) {
  const dustb_leaf_tables *T = c->mesh.leaf;
  L->n = 0;
  if (!global) {
    cand_push(L, m, 0, 0, 0);
    for (int k = 0; k < T->nnb[m]; ++k) {
      const int *s = &T->nbs[((size_t)m*DUSTB_LEAF_MAXNB + k)*3];
      cand_push(L, T->nb[(size_t)m*DUSTB_LEAF_MAXNB + k], s[0], s[1], s[2]);
    }
    return;
  }
  const int x3per = c->mesh.x3bc == 0;
  for (int b = 0; b < c->mesh.nmb; ++b) {
    int k0[3], k1[3];
    for (int a = 0; a < 3; ++a) {
      const int c0 = T->fbox[6*b + 2*a], c1 = T->fbox[6*b + 2*a + 1], n = T->nfine[a];
      k0[a] = fdiv(box[2*a] - (c1 + r), n) + 1;
      k1[a] = fdiv(box[2*a + 1] - (c0 - r), n);
    }
    if (!x3per) {
      if (k0[2] > 0 || k1[2] < 0) continue;
      k0[2] = k1[2] = 0;
    }
    for (int kz = k0[2]; kz <= k1[2]; ++kz)
      for (int ky = k0[1]; ky <= k1[1]; ++ky)
        for (int kx = k0[0]; kx <= k1[0]; ++kx) cand_push(L, b, -kx, -ky, -kz);
  }
}
static void cand_rect(const dustb_leaf_tables *T, const Cand *q, int r, int out[6]) {
  for (int a = 0; a < 3; ++a) {
    out[2*a] = T->fbox[6*q->b + 2*a] - q->s[a]*T->nfine[a] - r;
    out[2*a + 1] = T->fbox[6*q->b + 2*a + 1] - q->s[a]*T->nfine[a] + r;
  }
}
/* Meets: a candidate of level >= minlev, widened by r, meets the box */
static int leaf_meets(const dustb_ctx *c, int m, const int box[6], int minlev, int r,
                      int global) {
  const dustb_leaf_tables *T = c->mesh.leaf;
  CandList L = {NULL, 0, 0};
  candidates(c, m, global, box, r, &L);
  int hit = 0;
  for (int k = 0; k < L.n && !hit; ++k) {
    if (T->blev[L.v[k].b] < minlev) continue;
    int q[6];
    cand_rect(T, &L.v[k], r, q);
    hit = !(box[1] < q[0] || box[0] >= q[1] || box[3] < q[2] || box[2] >= q[3] ||
            box[5] < q[4] || box[4] >= q[5]);
  }
  free(L.v);
  return hit;
}
/* Covered: the band scan; each step takes, among the candidates holding the cell, the box
 * reaching furthest in x, then y, then z */
static int leaf_covered(const dustb_ctx *c, int m, const int box[6], int minlev, int r,
                        int global) {
  const dustb_leaf_tables *T = c->mesh.leaf;
  CandList L = {NULL, 0, 0};
  int ok = 1;
  int z = box[4];
  while (ok && z <= box[5]) {
    int ztop = box[5] + 1, y = box[2];
    while (ok && y <= box[3]) {
      int x = box[0], top = box[3] + 1;
      while (ok && x <= box[1]) {
        const int cell[6] = {x, x, y, y, z, z};
        candidates(c, m, global, cell, r, &L);
        int xe = x, ye = y, ze = z;
        for (int k = 0; k < L.n; ++k) {
          if (T->blev[L.v[k].b] < minlev) continue;
          int q[6];
          cand_rect(T, &L.v[k], r, q);
          if (x < q[0] || x >= q[1] || y < q[2] || y >= q[3] || z < q[4] || z >= q[5]) continue;
          if (q[1] > xe || (q[1] == xe && q[3] > ye) || (q[1] == xe && q[3] == ye && q[5] > ze)) {
            xe = q[1]; ye = q[3]; ze = q[5];
          }
        }
        if (xe == x) { ok = 0; break; }
        if (ye < top) top = ye;
        if (ze < ztop) ztop = ze;
        x = xe;
      }
      y = top;
    }
    z = ztop;
  }
  free(L.v);
  return ok;
}
static void leaf_clip_z(const dustb_ctx *c, int *ka, int *kb) {
  if (c->mesh.x3bc == 0) return;
  const int n = c->mesh.leaf->nfine[2];
  if (*ka < 0) *ka = 0;
  if (*kb > n - 1) *kb = n - 1;
}
static int leaf_need_global(const dustb_ctx *c, int m, const int box[6], int r) {
  const dustb_leaf_tables *T = c->mesh.leaf;
  int w[6] = {box[0] - r, box[1] + r, box[2] - r, box[3] + r, box[4] - r, box[5] + r};
  leaf_clip_z(c, &w[4], &w[5]);
  const int *f = &T->fbox[6*m], *sf = &T->safe[3*m];
  if (f[0] - sf[0] <= w[0] && f[1] + sf[0] > w[1] && f[2] - sf[1] <= w[2] &&
      f[3] + sf[1] > w[3] && f[4] - sf[2] <= w[4] && f[5] + sf[2] > w[5])
    return 0;
  return !leaf_covered(c, m, w, 0, 0, 0);
}

/* every leaf under the cloud `code` at the framed position x (anchor m) */
static void leaf_foreach(const dustb_ctx *c, const Ind *d, int m, const double x[3], int code,
                         int mom, CloudLeafFn f, void *ctx) {
  const dustb_mesh *ms = &c->mesh;
  const dustb_leaf_tables *T = ms->leaf;
  const double L[3] = {ms->x1max - ms->x1min, ms->x2max - ms->x2min, ms->x3max - ms->x3min};
  const int lev = code & 15, lb1 = (code >> 6) & 3, lb2 = (code >> 4) & 3, lb3 = (code >> 9) & 3;
  double h[3], ih[3];
  for (int a = 0; a < 3; ++a) { h[a] = ldexp(T->root_dx[a], -lev); ih[a] = ldexp(1.0/T->root_dx[a], lev); }
  Shape1 S[3];
  S[0] = make_shape(x[0], h[0], ih[0], lb1, mom);
  S[1] = make_shape(x[1], h[1], ih[1], lb2, mom);
  S[2] = make_shape(x[2], h[2], ih[2], lb3, mom);
  int npz = 1, zside = 0;
  if (ms->x3bc != 0 && (S[2].lo < ms->x3min || S[2].hi > ms->x3max)) {
    npz = 2; zside = S[2].hi > ms->x3max;
  }
  double fdx[3];
  for (int a = 0; a < 3; ++a) fdx[a] = T->root_dx[a]/(double)(1 << T->nlev);
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  CandList CL = {NULL, 0, 0};
  for (int part = 0; part < npz; ++part) {
    double zp = x[2];
    if (part == 1) {
      zp = 2.0*(zside ? ms->x3max : ms->x3min) - x[2];
      S[2] = make_shape(zp, h[2], ih[2], (lb3 == 1 || lb3 == 2) ? 3 - lb3 : lb3, mom);
    }
    int inside = 1;
    for (int a = 0; a < 3; ++a)
      inside = inside && S[a].lo >= MB(m, X1MIN + a) && S[a].hi <= MB(m, X1MIN + a) + nx[a]*MB(m, DX1 + a);
    CL.n = 0;
    if (inside) {
      cand_push(&CL, m, 0, 0, 0);
    } else {
      const double xmin[3] = {ms->x1min, ms->x2min, ms->x3min};
      int box[6];
      for (int a = 0; a < 3; ++a) {
        box[2*a] = (int)floor((S[a].lo - xmin[a])/fdx[a]);
        box[2*a + 1] = (int)ceil((S[a].hi - xmin[a])/fdx[a]) - 1;
      }
      leaf_clip_z(c, &box[4], &box[5]);
      const int global = leaf_need_global(c, m, box, 0);
      const int wide[6] = {box[0] - 1, box[1] + 1, box[2] - 1, box[3] + 1, box[4] - 1, box[5] + 1};
      CandList all = {NULL, 0, 0};
      candidates(c, m, global, wide, 0, &all);
      for (int k = 0; k < all.n; ++k) {
        const Cand *q = &all.v[k];
        int meets = 1;
        for (int a = 0; a < 3; ++a) {
          const double b0 = MB(q->b, X1MIN + a) - q->s[a]*L[a];
          meets = meets && !(S[a].hi <= b0 || S[a].lo >= b0 + nx[a]*MB(q->b, DX1 + a));
        }
        if (meets) cand_push(&CL, q->b, q->s[0], q->s[1], q->s[2]);
      }
      free(all.v);
    }
    for (int t = 0; t < CL.n; ++t) {
      const int b = CL.v[t].b;
      double o[3], dd[3];
      int lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        dd[a] = MB(b, DX1 + a);
        o[a] = MB(b, X1MIN + a) - CL.v[t].s[a]*L[a];
        const double id = 1.0/dd[a];
        lo[a] = (int)floor((S[a].lo - o[a])*id);
        hi[a] = (int)ceil((S[a].hi - o[a])*id) - 1;
        if (lo[a] < 0) lo[a] = 0;
        if (hi[a] > nx[a] - 1) hi[a] = nx[a] - 1;
      }
      for (int ic = lo[0]; ic <= hi[0]; ic += 4) {
        const int nr = (hi[0] - ic + 1 < 4) ? hi[0] - ic + 1 : 4;
        double w1[4] = {0.0, 0.0, 0.0, 0.0}, g1[4] = {0.0, 0.0, 0.0, 0.0};
        Face1 f1 = face_at(&S[0], o[0] + ic*dd[0], mom);
        for (int a = 0; a < nr; ++a) {
          const Face1 fn = face_at(&S[0], o[0] + (ic + a + 1)*dd[0], mom);
          cell_1d(&S[0], &f1, &fn, mom, &w1[a], &g1[a]);
          f1 = fn;
        }
        Face1 f3 = face_at(&S[2], o[2] + lo[2]*dd[2], mom);
        for (int k = lo[2]; k <= hi[2]; ++k) {
          const Face1 fn3 = face_at(&S[2], o[2] + (k + 1)*dd[2], mom);
          double w3, g3;
          cell_1d(&S[2], &f3, &fn3, mom, &w3, &g3);
          f3 = fn3;
          if (w3 == 0.0 && (!mom || g3 == 0.0)) continue;
          double czk = 0.0;
          if (mom && part == 1) {
            const double zc = o[2] + (k + 0.5)*dd[2];
            const double e = x[2] - zc;
            czk = (zp - zc) - (e - L[2]*round(e/L[2]));
          }
          Face1 f2 = face_at(&S[1], o[1] + lo[1]*dd[1], mom);
          for (int j = lo[1]; j <= hi[1]; ++j) {
            const Face1 fn2 = face_at(&S[1], o[1] + (j + 1)*dd[1], mom);
            double w2, g2;
            cell_1d(&S[1], &f2, &fn2, mom, &w2, &g2);
            f2 = fn2;
            if (w2 == 0.0 && (!mom || g2 == 0.0)) continue;
            const double w23 = w2*w3;
            for (int a = 0; a < nr; ++a) {
              CloudLeaf lf;
              lf.w = w23*w1[a];
              lf.m1x = lf.m1y = lf.m1z = 0.0;
              if (mom) {
                lf.m1x = w23*g1[a];
                lf.m1y = w1[a]*g2*w3;
                lf.m1z = w1[a]*w2*g3;
                if (part == 1) lf.m1z += czk*lf.w;
                if (lf.w == 0.0 && lf.m1x == 0.0 && lf.m1y == 0.0 && lf.m1z == 0.0) continue;
              } else if (lf.w == 0.0) {
                continue;
              }
              lf.b = b; lf.k = d->ks + k; lf.j = d->js + j; lf.i = d->is + ic + a;
              f(ctx, &lf);
            }
          }
        }
      }
    }
  }
  free(CL.v);
}

/* the leaf tables (DustGasDrag::BuildLeafTraversal3D, src/dust/dust_cloud3d.cpp:604-793), the
 * oracle's own build: geo nx1..3, nmb_root1..3, root_level, max_level, x3per; outputs as
 * dustb_host_leaf_tables.  The periodic shift of a neighbour: lround of the gap between the
 * facing sides across the slot's direction, of the centre offset along it, in domain lengths. */
int oracle_leaf_tables(const int *geo, int nmb, const int *lloc, const int *nghbr56, int *info,
                       int *fbox, int *blev, int *nnb, int *nb, int *nbs, int *nbmax, int *safe,
                       long long *lockey, int *locblk) {
  const int nlev = geo[7] - geo[6], x3per = geo[8];
  int nf[3];
  for (int a = 0; a < 3; ++a) nf[a] = (geo[3 + a]*geo[a]) << nlev;
  info[0] = nlev; info[1] = nf[0]; info[2] = nf[1]; info[3] = nf[2]; info[4] = 0;
  for (int b = 0; b < nmb; ++b) {
    blev[b] = lloc[4*b] - geo[6];
    for (int a = 0; a < 3; ++a) {
      fbox[6*b + 2*a] = (lloc[4*b + 1 + a]*geo[a]) << (nlev - blev[b]);
      fbox[6*b + 2*a + 1] = fbox[6*b + 2*a] + (geo[a] << (nlev - blev[b]));
    }
  }
  /* the direction of every slot, from the slot index formula of NeighborIndex */
  int dir[56][3];
  memset(dir, 0, sizeof(dir));
  for (int iz = -1; iz <= 1; ++iz)
    for (int iy = -1; iy <= 1; ++iy)
      for (int ix = -1; ix <= 1; ++ix) {
        const int nd = abs(ix) + abs(iy) + abs(iz);
        if (!nd) continue;
        for (int n2 = 0; n2 < 2; ++n2)
          for (int n1 = 0; n1 < 2; ++n1) {
            if ((nd >= 2 && n2) || (nd == 3 && n1)) continue;
            int s;
            if (iz == 0 && ix*iy == 0) s = abs(ix)*2*(ix + 1) + abs(iy)*2*(iy + 5) + n1 + 2*n2;
            else if (iz == 0) s = 16 + (ix + 1) + 2*(iy + 1) + n1;
            else if (ix*iy == 0) s = 24 + abs(ix)*(ix + 9) + abs(iy)*(iy + 17) + 2*(iz + 1) + n1 + 2*n2;
            else s = 48 + (ix + 1)/2 + (iy + 1) + 2*(iz + 1);
            dir[s][0] = ix; dir[s][1] = iy; dir[s][2] = iz;
          }
      }
  for (int m = 0; m < nmb; ++m) {
    int cnt = 0;
    for (int n = 0; n < 56; ++n) {
      const int b = nghbr56[56*m + n];
      if (b < 0) continue;
      int s[3];
      for (int a = 0; a < 3; ++a) {
        const double lo_b = fbox[6*b + 2*a], hi_b = fbox[6*b + 2*a + 1];
        const double lo_m = fbox[6*m + 2*a], hi_m = fbox[6*m + 2*a + 1];
        const double gap = dir[n][a] > 0 ? lo_b - hi_m
                         : (dir[n][a] < 0 ? hi_b - lo_m : 0.5*(lo_b + hi_b - lo_m - hi_m));
        s[a] = (int)lround(gap/nf[a]);
      }
      int seen = (b == m && !s[0] && !s[1] && !s[2]);
      for (int k = 0; k < cnt && !seen; ++k)
        seen = nb[m*DUSTB_LEAF_MAXNB + k] == b && nbs[(m*DUSTB_LEAF_MAXNB + k)*3] == s[0] &&
               nbs[(m*DUSTB_LEAF_MAXNB + k)*3 + 1] == s[1] && nbs[(m*DUSTB_LEAF_MAXNB + k)*3 + 2] == s[2];
      if (seen) continue;
      if (cnt >= DUSTB_LEAF_MAXNB) return -1;
      nb[m*DUSTB_LEAF_MAXNB + cnt] = b;
      for (int a = 0; a < 3; ++a) nbs[(m*DUSTB_LEAF_MAXNB + cnt)*3 + a] = s[a];
      ++cnt;
    }
    nnb[m] = cnt;
    for (int k = cnt; k < DUSTB_LEAF_MAXNB; ++k) {
      nb[m*DUSTB_LEAF_MAXNB + k] = -1;
      for (int a = 0; a < 3; ++a) nbs[(m*DUSTB_LEAF_MAXNB + k)*3 + a] = 0;
    }
  }
  for (int m = 0; m < nmb; ++m) {
    int mx = blev[m], w[3] = {0, 0, 0};
    for (int k = 0; k < nnb[m]; ++k) {
      const int b = nb[m*DUSTB_LEAF_MAXNB + k];
      if (blev[b] > mx) mx = blev[b];
      for (int a = 0; a < 3; ++a) {
        const int wd = fbox[6*b + 2*a + 1] - fbox[6*b + 2*a];
        if (k == 0 || wd < w[a]) w[a] = wd;
      }
    }
    nbmax[m] = mx;
    const int *f = &fbox[6*m];
    int ok = w[0] > 0 && w[1] > 0 && w[2] > 0;
    for (int a = 0; a < 3 && ok; ++a) ok = (f[2*a + 1] - f[2*a]) % w[a] == 0;
    for (int cz = f[4] - w[2]; ok && cz < f[5] + w[2]; cz += w[2])
      for (int cy = f[2] - w[1]; ok && cy < f[3] + w[1]; cy += w[1])
        for (int cx = f[0] - w[0]; ok && cx < f[1] + w[0]; cx += w[0]) {
          if (cx >= f[0] && cx < f[1] && cy >= f[2] && cy < f[3] && cz >= f[4] && cz < f[5]) continue;
          if (!x3per && (cz < 0 || cz >= nf[2])) continue;
          int held = 0;
          for (int k = 0; k < nnb[m] && !held; ++k) {
            const int b = nb[m*DUSTB_LEAF_MAXNB + k];
            const int *s = &nbs[(m*DUSTB_LEAF_MAXNB + k)*3];
            const int c3[3] = {cx, cy, cz};
            held = 1;
            for (int a = 0; a < 3; ++a)
              held = held && fbox[6*b + 2*a] - s[a]*nf[a] <= c3[a] &&
                     c3[a] + w[a] <= fbox[6*b + 2*a + 1] - s[a]*nf[a];
          }
          ok = held;
        }
    if (!ok) { w[0] = w[1] = w[2] = 0; ++info[4]; }
    for (int a = 0; a < 3; ++a) safe[3*m + a] = w[a];
  }
  /* the location index: keys ascending (insertion sort; the tests' meshes are small) */
  for (int b = 0; b < nmb; ++b) {
    const int sh = nlev - blev[b];
    const long long key = ((long long)blev[b] << 57) | ((long long)(fbox[6*b + 4]/(geo[2] << sh)) << 38) |
                          ((long long)(fbox[6*b + 2]/(geo[1] << sh)) << 19) |
                          (long long)(fbox[6*b]/(geo[0] << sh));
    int k = b;
    while (k > 0 && lockey[k - 1] > key) { lockey[k] = lockey[k - 1]; locblk[k] = locblk[k - 1]; --k; }
    lockey[k] = key; locblk[k] = b;
  }
  return 0;
}

/* Owner (src/dust/dust_leaf3d.hpp:534-595) without shear: the point framed next to block m (and
 * mirrored into the domain at a physical x3 face); the first of m and its neighbours whose box
 * holds it, else the block of Locate (:515-533, the location index level by level) */
static int leaf_owner(const dustb_ctx *c, const double px[3], int m) {
  const dustb_mesh *ms = &c->mesh;
  const dustb_leaf_tables *T = ms->leaf;
  const double L[3] = {ms->x1max - ms->x1min, ms->x2max - ms->x2min, ms->x3max - ms->x3min};
  const double xmin[3] = {ms->x1min, ms->x2min, ms->x3min};
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  double x[3] = {px[0], px[1], px[2]};
  for (int a = 0; a < (ms->x3bc == 0 ? 3 : 2); ++a) {
    const double cx = MB(m, X1MIN + a) + 0.5*nx[a]*MB(m, DX1 + a);
    x[a] -= L[a]*round((x[a] - cx)*(1.0/L[a]));
  }
  if (ms->x3bc != 0) {
    if (x[2] < ms->x3min) x[2] = 2.0*ms->x3min - x[2];
    if (x[2] >= ms->x3max) x[2] = fmin(2.0*ms->x3max - x[2], ms->x3max - 1.0e-12*L[2]);
  }
  CandList CL = {NULL, 0, 0};
  const int none[6] = {0, 0, 0, 0, 0, 0};
  candidates(c, m, 0, none, 0, &CL);
  int res = -1;
  for (int k = 0; k < CL.n && res < 0; ++k) {
    const int b = CL.v[k].b;
    int in = 1;
    for (int a = 0; a < 3; ++a) {
      const double fi = (x[a] - (MB(b, X1MIN + a) - CL.v[k].s[a]*L[a]))/MB(b, DX1 + a);
      in = in && fi >= 0.0 && fi < nx[a];
    }
    if (in) res = b;
  }
  free(CL.v);
  if (res >= 0) return res;
  int cc[3];
  for (int a = 0; a < 3; ++a) {
    const double fdx = T->root_dx[a]/(double)(1 << T->nlev);
    cc[a] = (int)floor((x[a] - xmin[a])/fdx);
    if (a == 2 && ms->x3bc != 0 && (cc[a] < 0 || cc[a] >= T->nfine[a])) return -1;
    cc[a] = ((cc[a] % T->nfine[a]) + T->nfine[a]) % T->nfine[a];
  }
  for (int l = 0; l <= T->nlev; ++l) {
    const int sh = T->nlev - l;
    const long long key = ((long long)l << 57) | ((long long)(cc[2]/(nx[2] << sh)) << 38) |
                          ((long long)(cc[1]/(nx[1] << sh)) << 19) | (long long)(cc[0]/(nx[0] << sh));
    for (int k = 0; k < ms->nmb; ++k)
      if (T->lockey[k] == key) return T->locblk[k];
  }
  return -1;
}

/* CloudInstantSwitch (src/dust/dust_cloud.cpp:1023-1085): every plain cloud of level >= L
 * takes max(L, the level of the block holding its centre); returns the clouds changed */
int oracle_cloud_instant_switch(const dustb_ctx *c, int L) {
  const dustb_mesh *ms = &c->mesh;
  if (L < 0 || L >= ms->leaf->nlev) return 0;
  const double *pr = c->part.pr; int *pi = c->part.pi; long long stride = c->part.stride;
  int n = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    const int code = PI(DUSTB_PLEV, p);
    if ((code & ~15) != 0 || code < L) continue;
    const double x[3] = {PR(DUSTB_IPX, p), PR(DUSTB_IPY, p), PR(DUSTB_IPZ, p)};
    int m = PI(DUSTB_PGID, p) - ms->gids;
    if (m < 0 || m >= ms->nmb) m = 0;
    const int b = leaf_owner(c, x, m);
    if (b < 0) continue;
    const int lev = ms->leaf->blev[b] > L ? ms->leaf->blev[b] : L;
    if (lev != code) { PI(DUSTB_PLEV, p) = lev; ++n; }
  }
  return n;
}

/* the split's eligibility (AnyAbove / AllAbove :596-622, SupportBox :653-666, InsideFiner
 * :668-681): the support of a plain level-lev cloud shrunk by the slack meets (overlap) or lies
 * on leaves above lev, the leaves of level l dilated by buffer << (nlev - l + 1) finest cells */
static int leaf_inside_finer(const dustb_ctx *c, const dustb_cloud_split *sp, double px,
                             double py, double pz, int lev, int m) {
  const dustb_mesh *ms = &c->mesh;
  const dustb_leaf_tables *T = ms->leaf;
  if (lev >= T->nlev || lev >= sp->max_level) return 0;
  if (sp->split_everywhere) return 1;
  const double L[3] = {ms->x1max - ms->x1min, ms->x2max - ms->x2min, ms->x3max - ms->x3min};
  const double xmin[3] = {ms->x1min, ms->x2min, ms->x3min};
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  double x[3] = {px, py, pz};
  for (int a = 0; a < (ms->x3bc == 0 ? 3 : 2); ++a) {
    const double cx = MB(m, X1MIN + a) + 0.5*nx[a]*MB(m, DX1 + a);
    x[a] -= L[a]*round((x[a] - cx)*(1.0/L[a]));
  }
  int box[6];
  for (int a = 0; a < 3; ++a) {
    const double r = (1.0 - sp->slack)*T->root_dx[a]/(double)(1 << lev);
    const double fdx = T->root_dx[a]/(double)(1 << T->nlev);
    box[2*a] = (int)floor((x[a] - r - xmin[a])/fdx);
    box[2*a + 1] = (int)ceil((x[a] + r - xmin[a])/fdx) - 1;
  }
  leaf_clip_z(c, &box[4], &box[5]);
  const int l1 = lev + 1;
  if (l1 > T->nlev) return 0;
  const int r = (sp->split_buffer > 0 && l1 >= 1 && l1 <= T->nlev) ? sp->split_buffer << (T->nlev - l1 + 1) : 0;
  const int g = leaf_need_global(c, m, box, r);
  if (!g && l1 > T->nbmax[m] && box[0] <= box[1] && box[2] <= box[3] && box[4] <= box[5]) return 0;
  return sp->split_overlap ? leaf_meets(c, m, box, l1, r, g) : leaf_covered(c, m, box, l1, r, g);
}
static double half_width(const dustb_leaf_tables *T, int lev, int a) {
  return T->root_dx[a]/(double)(1 << (lev & 15));
}
/* P1FlagT / P1SepT<LeafTraversal3D> (src/dust/dust_cloud3d.cpp:188-250) */
static int p1_flag(const dustb_ctx *c, const dustb_cloud_split *sp, int m, int code, const double x[3]) {
  const dustb_leaf_tables *T = c->mesh.leaf;
  const int lev = code & 15, l1 = (code >> 6) & 3, l2 = (code >> 4) & 3, l3 = (code >> 9) & 3;
  if (!l1 && !l2 && !l3) return leaf_inside_finer(c, sp, x[0], x[1], x[2], lev, m);
  if (lev > 0 && leaf_inside_finer(c, sp, x[0], x[1], x[2], lev - 1, m)) {
    const double h1 = half_width(T, lev - 1, 0), h2 = half_width(T, lev - 1, 1), h3 = half_width(T, lev - 1, 2);
    return ((l1 & 1) && leaf_inside_finer(c, sp, x[0] - h1, x[1], x[2], lev - 1, m)) ||
           ((l1 & 2) && leaf_inside_finer(c, sp, x[0] + h1, x[1], x[2], lev - 1, m)) ||
           ((l2 & 1) && leaf_inside_finer(c, sp, x[0], x[1] - h2, x[2], lev - 1, m)) ||
           ((l2 & 2) && leaf_inside_finer(c, sp, x[0], x[1] + h2, x[2], lev - 1, m)) ||
           ((l3 & 1) && leaf_inside_finer(c, sp, x[0], x[1], x[2] - h3, lev - 1, m)) ||
           ((l3 & 2) && leaf_inside_finer(c, sp, x[0], x[1], x[2] + h3, lev - 1, m));
  }
  return 0;
}
static int p1_sep(const dustb_ctx *c, const dustb_cloud_split *sp, int m, int code, const double x[3]) {
  const dustb_leaf_tables *T = c->mesh.leaf;
  const int lev = code & 15;
  const int l = ((code & ~15) == 0) ? lev : lev - 1;
  int s = 0;
  for (int a = 0; a < 3; ++a) {
    const double h = half_width(T, l, a);
    double lo[3] = {x[0], x[1], x[2]}, hi[3] = {x[0], x[1], x[2]};
    lo[a] -= h; hi[a] += h;
    if (leaf_inside_finer(c, sp, lo[0], lo[1], lo[2], l, m)) s |= 1 << (2*a);
    if (leaf_inside_finer(c, sp, hi[0], hi[1], hi[2], l, m)) s |= 2 << (2*a);
  }
  return s;
}
typedef struct { double off, frac; int lobe; } P1Piece;
/* P1Pieces3 (:52-65) */
static int p1_pieces(int lobe_old, int sep_lo, int sep_hi, P1Piece out[3]) {
  int n = 0;
  const double total = 0.5 + 0.25*((lobe_old & 1) ? 1 : 0) + 0.25*((lobe_old & 2) ? 1 : 0);
  const int lo = (lobe_old & 1) && sep_lo, hi = (lobe_old & 2) && sep_hi;
  const int lobe_new = lobe_old & ~((lo ? 1 : 0) | (hi ? 2 : 0));
  const double keep = 0.5 + 0.25*((lobe_new & 1) ? 1 : 0) + 0.25*((lobe_new & 2) ? 1 : 0);
  out[n].off = 0.0; out[n].frac = keep/total; out[n].lobe = lobe_new; ++n;
  if (lo) { out[n].off = -1.0; out[n].frac = 0.25/total; out[n].lobe = 0; ++n; }
  if (hi) { out[n].off = 1.0; out[n].frac = 0.25/total; out[n].lobe = 0; ++n; }
  return n;
}
static double wrap_pos(double x, double lo, double hi) {
  const double len = hi - lo;
  while (x < lo) x += len;
  while (x >= hi) x -= len;
  return x;
}
/* SplitCloudsP1DeviceT (src/dust/dust_cloud3d.cpp:1005-1310) without the split velocity and
 * the block marks: the count pass, the exclusive scan of the appended pieces, the
 * fill (pieces last to first, the parent's slot last).  The arrays must hold npart + the pieces;
 * returns the pieces appended (npart is not changed), or -1 when they exceed the capacity. */
int oracle_cloud_split_p1(const dustb_ctx *c, const dustb_cloud_split *sp, unsigned long long tag0) {
  const dustb_mesh *ms = &c->mesh;
  const dustb_leaf_tables *T = ms->leaf;
  double *pr = c->part.pr; int *pi = c->part.pi; long long stride = c->part.stride;
  const int np = c->part.npart;
  int *sep = (int *)calloc((size_t)np + 1, sizeof(int));
  int *off = (int *)calloc((size_t)np + 1, sizeof(int));
  int total = 0;
  for (int p = 0; p < np; ++p) {
    const int code = PI(DUSTB_PLEV, p);
    const double x[3] = {PR(DUSTB_IPX, p), PR(DUSTB_IPY, p), PR(DUSTB_IPZ, p)};
    int m = PI(DUSTB_PGID, p) - ms->gids;
    if (m < 0 || m >= ms->nmb) m = 0;
    off[p] = total;
    if ((code & ~(15 | (3 << 4) | (3 << 6) | (3 << 9))) != 0 || !p1_flag(c, sp, m, code, x)) continue;
    const int s = p1_sep(c, sp, m, code, x);
    const int plain = (code & ~15) == 0;
    P1Piece pc[3][3];
    int n = 1;
    for (int a = 0; a < 3; ++a) {
      const int lobe = plain ? 3 : ((a == 0) ? (code >> 6) & 3 : ((a == 1) ? (code >> 4) & 3 : (code >> 9) & 3));
      n *= p1_pieces(lobe, (s >> (2*a)) & 1, (s >> (2*a + 1)) & 1, pc[a]);
    }
    sep[p] = s | 64;
    total += n - 1;
  }
  if (sp->budget > 0 && (long long)total > sp->budget) {
    /* the split budget (:1062-1111): events whose pieces start at or beyond it wait */
    int taken = total;
    for (int p = 0; p < np; ++p)
      if (sep[p] && (long long)off[p] >= sp->budget) {
        sep[p] = 0;
        if (off[p] < taken) taken = off[p];
      }
    total = taken;
  }
  if ((long long)np + total > stride) { free(sep); free(off); return -1; }
  const int reflect = ms->x3bc == 1;
  for (int p = 0; p < np; ++p) {
    if (!sep[p]) continue;
    const int code = PI(DUSTB_PLEV, p);
    const int lev = code & 15, plain = (code & ~15) == 0;
    const double x[3] = {PR(DUSTB_IPX, p), PR(DUSTB_IPY, p), PR(DUSTB_IPZ, p)};
    const double mass = PR(DUSTB_IPM, p);
    P1Piece pc[3][3];
    int n[3];
    for (int a = 0; a < 3; ++a) {
      const int lobe = plain ? 3 : ((a == 0) ? (code >> 6) & 3 : ((a == 1) ? (code >> 4) & 3 : (code >> 9) & 3));
      n[a] = p1_pieces(lobe, (sep[p] >> (2*a)) & 1, (sep[p] >> (2*a + 1)) & 1, pc[a]);
    }
    const int clev = plain ? lev + 1 : lev;
    double e[3];
    for (int a = 0; a < 3; ++a) e[a] = half_width(T, clev, a);
    const int n12 = n[0]*n[1];
    for (int k = n12*n[2] - 1; k >= 0; --k) {
      const int ia[3] = {k % n[0], (k/n[0]) % n[1], k/n12};
      const int s = (k == 0) ? p : np + off[p] + k - 1;
      double cpos[3];
      for (int a = 0; a < 3; ++a) cpos[a] = x[a] + pc[a][ia[a]].off*e[a];
      int zmir = 0;
      cpos[0] = wrap_pos(cpos[0], ms->x1min, ms->x1max);
      cpos[1] = wrap_pos(cpos[1], ms->x2min, ms->x2max);
      if (ms->x3bc == 0) {
        cpos[2] = wrap_pos(cpos[2], ms->x3min, ms->x3max);
      } else if (cpos[2] < ms->x3min) {
        cpos[2] = 2.0*ms->x3min - cpos[2]; zmir = 1;
      } else if (cpos[2] >= ms->x3max) {
        cpos[2] = 2.0*ms->x3max - cpos[2]; zmir = 1;
        if (cpos[2] >= ms->x3max) cpos[2] = ms->x3max - 1.0e-12*(ms->x3max - ms->x3min);
      }
      if (k > 0) {
        for (int q = 0; q < DUSTB_NREAL; ++q) PR(q, s) = PR(q, p);
        for (int q = 0; q < DUSTB_NINT; ++q) PI(q, s) = PI(q, p);
        const unsigned long long t = tag0 + (unsigned long long)(off[p] + k - 1);
        PI(DUSTB_PTAG, s) = (int)(unsigned)(t & 0xffffffffULL);
        PI(DUSTB_PTAGH, s) = (int)(unsigned)(t >> 32);
      }
      PR(DUSTB_IPX, s) = cpos[0]; PR(DUSTB_IPX1, s) = cpos[0];
      PR(DUSTB_IPY, s) = cpos[1]; PR(DUSTB_IPY1, s) = cpos[1];
      PR(DUSTB_IPZ, s) = cpos[2]; PR(DUSTB_IPZ1, s) = cpos[2];
      double mp = mass*pc[0][ia[0]].frac*pc[1][ia[1]].frac;
      mp = mp*pc[2][ia[2]].frac;
      const int l3 = pc[2][ia[2]].lobe;
      PR(DUSTB_IPM, s) = mp;
      PI(DUSTB_PLEV, s) = clev | (pc[0][ia[0]].lobe << 6) | (pc[1][ia[1]].lobe << 4) |
                          ((zmir && (l3 == 1 || l3 == 2) ? 3 - l3 : l3) << 9);
      if (zmir && reflect) { PR(DUSTB_IPVZ, s) = -PR(DUSTB_IPVZ, s); PR(DUSTB_IPVZ1, s) = -PR(DUSTB_IPVZ1, s); }
      int am = PI(DUSTB_PGID, s) - ms->gids;
      if (am < 0 || am >= ms->nmb) am = 0;
      const int b = leaf_owner(c, cpos, am);
      PI(DUSTB_PGID, s) = ms->gids + ((b >= 0 && b < ms->nmb) ? b : am);
    }
  }
  free(sep); free(off);
  return total;
}

/* every leaf of the cloud at x (level code, anchored at block m): f(ctx, leaf); with moments the
 * moment traversal, else the weight traversal */
static void cloud_leaves(const dustb_ctx *c, const Ind *d, int m, const double x[3], int code,
                         int moments, CloudLeafFn f, void *ctx, unsigned *err) {
  const dustb_mesh *ms = &c->mesh;
  if (ms->leaf) { leaf_foreach(c, d, m, x, code, moments, f, ctx); return; }
  const double Lz = ms->x3max - ms->x3min;
  CloudAxis X, Y, Z;
  cloud_axis(c, m, 0, x[0], code, &X);
  cloud_axis(c, m, 1, x[1], code, &Y);
  if (ms->three_d) cloud_axis(c, m, 2, x[2], code, &Z);
  else { Z.n = 1; Z.o[0] = 0; Z.i[0] = 0; Z.w[0] = 1.0; Z.g[0] = 0.0; Z.org[0] = 0.0; }
  int npz = 1;
  double zp = x[2];
  if (ms->three_d && ms->x3bc != 0) {
    const double ell = ldexp(MB(m, DX3), -code);
    const double lo = x[2] - ell, hi = x[2] + ell;
    if (lo < ms->x3min || hi > ms->x3max) {
      npz = 2;
      zp = 2.0*((hi > ms->x3max) ? ms->x3max : ms->x3min) - x[2];
    }
  }
  for (int part = 0; part < npz; ++part) {
    if (part == 1) cloud_axis(c, m, 2, zp, code, &Z);
    for (int kz = 0; kz < Z.n; ++kz) {
      const double w3 = Z.w[kz], g3 = Z.g[kz];
      if (w3 == 0.0 && (!moments || g3 == 0.0)) continue;
      double czk = 0.0;
      if (moments && part == 1) {
        const double zc = Z.org[kz] + (Z.i[kz] + 0.5)*MB(m, DX3);
        const double ez = x[2] - zc;
        czk = (zp - zc) - (ez - Lz*round(ez/Lz));
      }
      for (int jy = 0; jy < Y.n; ++jy) {
        const double w2 = Y.w[jy], g2 = Y.g[jy];
        if (w2 == 0.0 && (!moments || g2 == 0.0)) continue;
        const double w23 = w2*w3;
        for (int ix = 0; ix < X.n; ++ix) {
          const double wa = X.w[ix];
          CloudLeaf lf;
          lf.w = w23*wa;
          lf.m1x = lf.m1y = lf.m1z = 0.0;
          if (moments) {
            lf.m1x = w23*X.g[ix];
            lf.m1y = wa*g2*w3;
            lf.m1z = wa*w2*g3;
            if (part == 1) lf.m1z += czk*lf.w;
            if (lf.w == 0.0 && lf.m1x == 0.0 && lf.m1y == 0.0 && lf.m1z == 0.0) continue;
          } else if (lf.w == 0.0) {
            continue;
          }
          lf.b = cloud_owner(c, m, X.o[ix], Y.o[jy], Z.o[kz]);
          if (lf.b < 0) { if (err) *err |= DUSTB_ERR_CLOUD; continue; }
          lf.k = d->ks + Z.i[kz]; lf.j = d->js + Y.i[jy]; lf.i = d->is + X.i[ix];
          f(ctx, &lf);
        }
      }
    }
  }
}

/* ---- the linear gather and the deposits, as callbacks ---- */
typedef struct {
  const dustb_ctx *c; const Ind *d; const double *x; const double *gp; double ug[3];
} GatherCtx;
static void gather_leaf(void *vctx, const CloudLeaf *lf) {
  GatherCtx *g = (GatherCtx *)vctx;
  const dustb_ctx *c = g->c; const dustb_mesh *ms = &c->mesh; const Ind *d = g->d;
  const double L[3] = {ms->x1max - ms->x1min, ms->x2max - ms->x2min, ms->x3max - ms->x3min};
  const int b = lf->b;
  const double w = lf->w;
  const double dx1 = MB(b, DX1), dx2 = MB(b, DX2), dx3 = MB(b, DX3);
  const double xc = MB(b, X1MIN) + (lf->i - d->is + 0.5)*dx1;
  const double yc = MB(b, X2MIN) + (lf->j - d->js + 0.5)*dx2;
  const double ex = g->x[0] - xc, ey = g->x[1] - yc;
  const double cx = 0.5*(lf->m1x + (ex - L[0]*round(ex/L[0]))*w)/dx1;
  const double cy = 0.5*(lf->m1y + (ey - L[1]*round(ey/L[1]))*w)/dx2;
  const double *gp = g->gp + ((((size_t)b*d->n3 + lf->k)*d->n2 + lf->j)*d->n1 + lf->i)*12;
  if (ms->three_d) {
    const double zc = MB(b, X3MIN) + (lf->k - d->ks + 0.5)*dx3;
    const double ez = g->x[2] - zc;
    const double cz = 0.5*(lf->m1z + (ez - L[2]*round(ez/L[2]))*w)/dx3;
    g->ug[0] += w*gp[0] + cx*gp[3] + cy*gp[6] + cz*gp[9];
    g->ug[1] += w*gp[1] + cx*gp[4] + cy*gp[7] + cz*gp[10];
    g->ug[2] += w*gp[2] + cx*gp[5] + cy*gp[8] + cz*gp[11];
  } else {
    g->ug[0] += w*gp[0] + cx*gp[3] + cy*gp[6];
    g->ug[1] += w*gp[1] + cx*gp[4] + cy*gp[7];
    g->ug[2] += w*gp[2] + cx*gp[5] + cy*gp[8];
  }
}
/* the clouds' linear gather of the packed field gp at one cloud (CloudLinearGather3D without
 * the blend) */
static void cloud_gather(const dustb_ctx *c, const Ind *d, int m, const double x[3], int code,
                         const double *gp, double ug[3], unsigned *err) {
  GatherCtx g = {c, d, x, gp, {0.0, 0.0, 0.0}};
  cloud_leaves(c, d, m, x, code, 1, gather_leaf, &g, err);
  ug[0] = g.ug[0]; ug[1] = g.ug[1]; ug[2] = g.ug[2];
}

/* s * w / V * v[q] into f(b, nvar, c0 + q) for q < n: the deposits of the cloud kernels */
typedef struct {
  const dustb_ctx *c; const Ind *d; double *f; int nvar, c0, n; double s; double v[4];
  int inv_first;   /* 1: (1 / V) w v (the pc2 predictor's product order), 0: s w / V v */
} DepositCtx;
static void deposit_leaf(void *vctx, const CloudLeaf *lf) {
  DepositCtx *q = (DepositCtx *)vctx;
  const Ind *d = q->d;
  if (q->inv_first) {
    const double inv_volume = 1.0/cloud_measure(q->c, lf->b);
    for (int t = 0; t < q->n; ++t)
      A5(q->f, q->nvar, (*d), lf->b, q->c0 + t, lf->k, lf->j, lf->i) += inv_volume*lf->w*q->v[t];
  } else {
    const double dw = q->s*lf->w/cloud_measure(q->c, lf->b);
    for (int t = 0; t < q->n; ++t)
      A5(q->f, q->nvar, (*d), lf->b, q->c0 + t, lf->k, lf->j, lf->i) += dw*q->v[t];
  }
}
static void cloud_deposit(const dustb_ctx *c, const Ind *d, int m, const double x[3], int code,
                          double *f, int nvar, int c0, int n, double s, const double *v,
                          int inv_first, unsigned *err) {
  DepositCtx q = {c, d, f, nvar, c0, n, s, {0.0, 0.0, 0.0, 0.0}, inv_first};
  for (int t = 0; t < n; ++t) q.v[t] = v[t];
  cloud_leaves(c, d, m, x, code, 0, deposit_leaf, &q, err);
}

/* CloudDepositImplicitT (src/dust/dust_imex3d.cpp:61-99): Q = m c W / V and P = Q v into
 * qdep 0-3 of the owner cells (qdep cleared first) */
unsigned oracle_cloud_deposit_qp(const dustb_ctx *c, double a_dt, double sh) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  memset(c->f.qdep, 0, field_size(ms, 5)*sizeof(double));
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  unsigned err = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    const int m = PI(DUSTB_PGID, p) - ms->gids;
    const int code = PI(DUSTB_PLEV, p);
    double x[3];
    cloud_position(c, p, sh, x);
    if (!cloud_frame_ok(c, m, x, code, 0.0)) { err |= DUSTB_ERR_CLOUD; continue; }
    const double mass_c = ms->three_d ? PR(DUSTB_IPM, p)*a_dt/(PR(DUSTB_IPTS, p) + a_dt)
                                      : PR(DUSTB_IPM, p)*(a_dt/(PR(DUSTB_IPTS, p) + a_dt));
    const double v[4] = {1.0, PR(DUSTB_IPVX, p), PR(DUSTB_IPVY, p), PR(DUSTB_IPVZ, p)};
    /* (dw = m c w / V, then dw, dw vx, dw vy, dw vz: the factor 1 keeps dw itself) */
    cloud_deposit(c, &d, m, x, code, c->f.qdep, 5, 0, 4, mass_c, v, 0, &err);
  }
  return err;
}

/* PackGatherField3D (src/dust/dust_cloud3d.cpp:1319-1340): gp(m, k, j, i, 0..11) = the
 * velocity and its central differences along x, y, z, over the padded interior; 2-D
 * (PackGatherField, src/dust/dust_pm.cpp:81-102): the plane ks, no x3 differences */
void oracle_gather_pack(const dustb_ctx *c, const double *v, double *gp) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  memset(gp, 0, (size_t)ms->nmb*d.n3*d.n2*d.n1*12*sizeof(double));
  const int k0 = ms->three_d ? 1 : d.ks, k1 = ms->three_d ? d.n3 - 2 : d.ks;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = k0; k <= k1; ++k)
      for (int j = 1; j < d.n2 - 1; ++j)
        for (int i = 1; i < d.n1 - 1; ++i) {
          double *g = gp + ((((size_t)m*d.n3 + k)*d.n2 + j)*d.n1 + i)*12;
          for (int q = 0; q < 3; ++q) {
            g[q] = A5(v, 3, d, m, q, k, j, i);
            g[3 + q] = A5(v, 3, d, m, q, k, j, i + 1) - A5(v, 3, d, m, q, k, j, i - 1);
            g[6 + q] = A5(v, 3, d, m, q, k, j + 1, i) - A5(v, 3, d, m, q, k, j - 1, i);
            if (ms->three_d)
              g[9 + q] = A5(v, 3, d, m, q, k + 1, j, i) - A5(v, 3, d, m, q, k - 1, j, i);
          }
        }
}

/* CloudGatherKickT without the blend (src/dust/dust_imex3d.cpp:114-175, the linear gather
 * CloudLinearGather3D / GatherLinear, src/dust/dust_imex3d_gather.hpp, dust_leaf_api.hpp:
 * 196-219): ubar = sum over the leaves of w u* + cx du/dx + cy du/dy + cz du/dz with
 * cx = (m1x + MinImage(x - xc) w) / (2 dx); dv = c (ubar - v), v += dv, R = dv / a_dt; with
 * back-reaction -m w dv / V into dmom (cleared first) of the leaves of nonzero weight.  gp: the
 * pack of u* (its ghost cells filled by the caller). */
unsigned oracle_cloud_gather_kick(const dustb_ctx *c, double a_dt, double sh, const double *gp) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  memset(c->f.dmom, 0, field_size(ms, 3)*sizeof(double));
  double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int br = c->phys.back_reaction;
  unsigned err = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    const int m = PI(DUSTB_PGID, p) - ms->gids;
    const int code = PI(DUSTB_PLEV, p);
    double x[3];
    cloud_position(c, p, sh, x);
    if (!cloud_frame_ok(c, m, x, code, 0.0)) { err |= DUSTB_ERR_CLOUD; continue; }
    double ug[3];
    cloud_gather(c, &d, m, x, code, gp, ug, &err);
    const double cj = a_dt/(PR(DUSTB_IPTS, p) + a_dt);
    const double dvx = cj*(ug[0] - PR(DUSTB_IPVX, p));
    const double dvy = cj*(ug[1] - PR(DUSTB_IPVY, p));
    const double dvz = cj*(ug[2] - PR(DUSTB_IPVZ, p));
    PR(DUSTB_IPVX, p) += dvx; PR(DUSTB_IPVY, p) += dvy; PR(DUSTB_IPVZ, p) += dvz;
    PR(DUSTB_IPRX, p) = dvx/a_dt; PR(DUSTB_IPRY, p) = dvy/a_dt; PR(DUSTB_IPRZ, p) = dvz/a_dt;
    if (!br) continue;
    const double v[3] = {dvx, dvy, dvz};
    cloud_deposit(c, &d, m, x, code, c->f.dmom, 3, 0, 3, -PR(DUSTB_IPM, p), v, 0, NULL);
  }
  return err;
}

/* the clouds' copy exchanges: on a refined mesh the multilevel one (its coarse arrays
 * allocated here) */
void oracle_ghost_copy_ml(const dustb_ctx *c, double *a, int nvar, double *ca);
static void cloud_copy_exchange(const dustb_ctx *c, double *a, int nvar, int x3_bcs) {
  const dustb_mesh *ms = &c->mesh;
  if (!ms->nghbr_ml) { oracle_ghost_copy(c, a, nvar, x3_bcs); return; }
  const size_t n = (size_t)ms->nmb*nvar*(ms->nx1/2 + 2*ms->ng)*(ms->nx2/2 + 2*ms->ng)*
                   (ms->nx3/2 + 2*ms->ng);
  double *ca = (double *)malloc(n*sizeof(double));
  oracle_ghost_copy_ml(c, a, nvar, ca);
  free(ca);
}

/* CloudDefectCorrection (src/dust/dust_imex3d_dc.cpp:229-274) with CloudOperatorKernelT
 * (dust_cloud_imex_kernels.hpp:20-70): one sweep x <- x + (rho + Q)^-1 (M + P - rho x - D M G x)
 * on u*, the operator D M G x = the clouds' m c W ubar / V with ubar their linear gather of x
 * (u*'s ghost cells by the copy exchange first; the operator's result in work) */
unsigned oracle_cloud_dc1_sweep(const dustb_ctx *c, double a_dt, double sh) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  double *x = c->f.ustar, *r = c->f.work;
  double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  cloud_copy_exchange(c, x, 3, 1);
  double *gp = (double *)malloc((size_t)ms->nmb*d.n3*d.n2*d.n1*12*sizeof(double));
  oracle_gather_pack(c, x, gp);
  memset(r, 0, field_size(ms, 3)*sizeof(double));
  unsigned err = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    const int m = PI(DUSTB_PGID, p) - ms->gids;
    const int code = PI(DUSTB_PLEV, p);
    double xp[3];
    cloud_position(c, p, sh, xp);
    if (!cloud_frame_ok(c, m, xp, code, 0.0)) { err |= DUSTB_ERR_CLOUD; continue; }
    double ug[3];
    cloud_gather(c, &d, m, xp, code, gp, ug, &err);
    const double mc = PR(DUSTB_IPM, p)*(a_dt/(PR(DUSTB_IPTS, p) + a_dt));
    cloud_deposit(c, &d, m, xp, code, r, 3, 0, 3, mc, ug, 0, NULL);
  }
  free(gp);
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i) {
          const double rho = A5(c->f.u0, nv, d, m, 0, k, j, i);
          const double pinv = 1.0/(rho + A5(c->f.qdep, 5, d, m, 0, k, j, i));
          for (int v = 0; v < 3; ++v) {
            const double av = A5(r, 3, d, m, v, k, j, i) + rho*A5(x, 3, d, m, v, k, j, i);
            const double rv = A5(c->f.u0, nv, d, m, 1 + v, k, j, i) +
                              A5(c->f.qdep, 5, d, m, 1 + v, k, j, i) - av;
            A5(x, 3, d, m, v, k, j, i) += pinv*rv;
          }
        }
  return err;
}

/* the overlap split's particle part: rv = sum over the leaves of w res */
typedef struct { const Ind *d; const double *res; double rv[3]; } ResCtx;
static void res_leaf(void *vctx, const CloudLeaf *lf) {
  ResCtx *q = (ResCtx *)vctx;
  for (int v = 0; v < 3; ++v) q->rv[v] += lf->w*A5(q->res, 4, (*q->d), lf->b, v, lf->k, lf->j, lf->i);
}

/* ApplyPMBR for the clouds (src/dust/dust_pm.cpp:576-711): with imex_consistent_gas the
 * overlap split CloudImplicitConsistencyOverlapT (src/dust/dust_imex3d.cpp:669-790): per cell
 * g = rho u* - M, r = (D - g) / (rho + Q), the gas takes g + rho r and dmom its rate; every
 * cloud v += c sum W r, R += c sum W r / a_dt with the deposit's weights.  Otherwise the plain
 * PMBR of the points. */
void oracle_cloud_apply_pmbr(const dustb_ctx *c, double a_dt, double sh) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  if (!c->phys.back_reaction) return;
  if (!c->phys.consistent_gas) { oracle_apply_pmbr(c, a_dt); return; }
  const double inv_adt = 1.0/a_dt;
  double *u0 = c->f.u0, *dm = c->f.dmom, *res = c->f.resid;
  memset(res, 0, field_size(ms, 4)*sizeof(double));
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i) {
          const double rho = A5(u0, nv, d, m, 0, k, j, i);
          const double q = A5(c->f.qdep, 5, d, m, 0, k, j, i);
          const double inv = 1.0/(rho + q);
          for (int v = 0; v < 3; ++v) {
            const double g = rho*A5(c->f.ustar, 3, d, m, v, k, j, i) - A5(u0, nv, d, m, 1 + v, k, j, i);
            const double r = (A5(dm, 3, d, m, v, k, j, i) - g)*inv;
            const double dgas = g + rho*r;
            A5(u0, nv, d, m, 1 + v, k, j, i) += dgas;
            A5(dm, 3, d, m, v, k, j, i) = dgas*inv_adt;
            A5(res, 4, d, m, v, k, j, i) = r;
          }
        }
  double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  for (int p = 0; p < c->part.npart; ++p) {
    if (PR(DUSTB_IPM, p) <= 0.0) continue;
    const int m = PI(DUSTB_PGID, p) - ms->gids;
    const int code = PI(DUSTB_PLEV, p);
    double x[3];
    cloud_position(c, p, sh, x);
    if (!cloud_frame_ok(c, m, x, code, 0.0)) continue;
    ResCtx q = {&d, res, {0.0, 0.0, 0.0}};
    cloud_leaves(c, &d, m, x, code, 0, res_leaf, &q, NULL);
    const double cj = a_dt/(PR(DUSTB_IPTS, p) + a_dt);
    PR(DUSTB_IPVX, p) += cj*q.rv[0]; PR(DUSTB_IPVY, p) += cj*q.rv[1]; PR(DUSTB_IPVZ, p) += cj*q.rv[2];
    PR(DUSTB_IPRX, p) += cj*q.rv[0]/a_dt; PR(DUSTB_IPRY, p) += cj*q.rv[1]/a_dt;
    PR(DUSTB_IPRZ, p) += cj*q.rv[2]/a_dt;
  }
}

/* ---- the clouds' pc2 (src/dust/dust_cloud3d.cpp:1362-1538, CloudPC2Push :76-150) ------- */
/* CloudPredictorT: the step-start gas velocity (PackGasGather3D: u1 momentum over density in
 * every cell, then packed) gathered linearly over the cloud; g = -dt (m / t_s) (ubar - v) into
 * qdep 1-3 and, with rate_dep, m / t_s into qdep 4, with the cloud's weights (qdep cleared) */
unsigned oracle_cloud_pc2_predictor(const dustb_ctx *c, double dt, int rate_dep) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  memset(c->f.qdep, 0, field_size(ms, 5)*sizeof(double));
  double *uv = (double *)malloc(field_size(ms, 3)*sizeof(double));
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = 0; k < d.n3; ++k)
      for (int j = 0; j < d.n2; ++j)
        for (int i = 0; i < d.n1; ++i) {
          const double invrho = 1.0/A5(c->f.u1, nv, d, m, 0, k, j, i);
          for (int v = 0; v < 3; ++v)
            A5(uv, 3, d, m, v, k, j, i) = A5(c->f.u1, nv, d, m, 1 + v, k, j, i)*invrho;
        }
  double *gp = (double *)malloc((size_t)ms->nmb*d.n3*d.n2*d.n1*12*sizeof(double));
  oracle_gather_pack(c, uv, gp);
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  unsigned err = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    const int m = PI(DUSTB_PGID, p) - ms->gids;
    const int code = PI(DUSTB_PLEV, p);
    double x[3];
    cloud_position(c, p, 0.0, x);
    if (!cloud_frame_ok(c, m, x, code, 0.0)) { err |= DUSTB_ERR_CLOUD; continue; }
    double ug[3];
    cloud_gather(c, &d, m, x, code, gp, ug, &err);
    const double mass_rate = PR(DUSTB_IPM, p)/PR(DUSTB_IPTS, p);
    const double v[4] = {-dt*mass_rate*(ug[0] - PR(DUSTB_IPVX, p)),
                         -dt*mass_rate*(ug[1] - PR(DUSTB_IPVY, p)),
                         -dt*mass_rate*(ug[2] - PR(DUSTB_IPVZ, p)), mass_rate};
    cloud_deposit(c, &d, m, x, code, c->f.qdep, 5, 1, rate_dep ? 4 : 3, 1.0, v, 1, NULL);
  }
  free(gp); free(uv);
  return err;
}

/* CloudAdvanceT: from the stage-start registers (X1, V1) the midpoint xh and the gather
 * position xg (CloudPC2Push::Midpoint), ubar = the linear gather of u* (ghost cells filled by the
 * caller) at xg, the implicit-midpoint kick (Kick: the 2x2 Coriolis solve, vertical gravity),
 * v = 2 vh - v0, the drift, X1 = xh, R = dt (ubar - vh) / t_s, and with back-reaction -m W R / V
 * into dmom (cleared) */
unsigned oracle_cloud_pc2_advance(const dustb_ctx *c, double dt) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  memset(c->f.dmom, 0, field_size(ms, 3)*sizeof(double));
  double *gp = (double *)malloc((size_t)ms->nmb*d.n3*d.n2*d.n1*12*sizeof(double));
  oracle_gather_pack(c, c->f.ustar, gp);
  double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int br = c->phys.back_reaction, sbox = c->phys.shearing_box, strat = c->phys.stratified;
  const double q = c->phys.qshear, om = c->phys.omega0, aphi = c->phys.const_accel_phi;
  unsigned err = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    const int m = PI(DUSTB_PGID, p) - ms->gids;
    const double x0[3] = {PR(DUSTB_IPX1, p), PR(DUSTB_IPY1, p), ms->three_d ? PR(DUSTB_IPZ1, p) : 0.0};
    const double v0[3] = {PR(DUSTB_IPVX1, p), PR(DUSTB_IPVY1, p), PR(DUSTB_IPVZ1, p)};
    double xh[3], xg[3];
    if (ms->three_d) {
      xh[0] = x0[0] + 0.5*dt*v0[0];
      xh[1] = x0[1] + 0.5*dt*(v0[1] - (sbox ? q*om*x0[0] : 0.0));
      xh[2] = x0[2] + 0.5*dt*v0[2];
      xg[0] = xh[0];
      xg[1] = xh[1] + (sbox ? q*om*xh[0]*0.5*dt : 0.0);
      xg[2] = xh[2];
    } else {
      xh[0] = x0[0] + 0.5*dt*v0[0];
      xh[1] = x0[1] + 0.5*dt*v0[1];
      xh[2] = x0[2];
      xg[0] = xh[0]; xg[1] = xh[1]; xg[2] = xh[2];
    }
    const int code = PI(DUSTB_PLEV, p);
    double xf[3] = {xg[0], xg[1], xg[2]};
    if (!cloud_frame_ok(c, m, xf, code, 1.0)) { err |= DUSTB_ERR_CLOUD; continue; }
    double ug[3];
    cloud_gather(c, &d, m, xf, code, gp, ug, &err);
    const double h = 0.5*dt;
    const double lambda = h/PR(DUSTB_IPTS, p);
    const double aa = 1.0 + lambda;
    double r[3] = {v0[0] + lambda*ug[0], v0[1] + lambda*ug[1], v0[2] + lambda*ug[2]};
    double vh[3];
    if (ms->three_d) {
      if (sbox) {
        const double cxy = 2.0*h*om, cyx = h*(2.0 - q)*om;
        const double det = aa*aa + cxy*cyx;
        vh[0] = (aa*r[0] + cxy*r[1])/det;
        vh[1] = (aa*r[1] - cyx*r[0])/det;
        if (strat) r[2] -= h*(om*om)*xh[2];
        vh[2] = r[2]/aa;
      } else {
        vh[0] = r[0]/aa; vh[1] = r[1]/aa; vh[2] = r[2]/aa;
      }
    } else {
      if (sbox) {
        const double cxz = 2.0*h*om, czx = h*(2.0 - q)*om;
        const double det = aa*aa + cxz*czx;
        if (aphi != 0.0) r[2] += h*aphi;
        vh[0] = (aa*r[0] + cxz*r[2])/det;
        vh[2] = (aa*r[2] - czx*r[0])/det;
        vh[1] = r[1]/aa;
      } else {
        vh[0] = r[0]/aa; vh[1] = r[1]/aa; vh[2] = r[2]/aa;
      }
    }
    PR(DUSTB_IPVX, p) = 2.0*vh[0] - v0[0];
    PR(DUSTB_IPVY, p) = 2.0*vh[1] - v0[1];
    PR(DUSTB_IPVZ, p) = 2.0*vh[2] - v0[2];
    PR(DUSTB_IPX, p) = x0[0] + dt*vh[0];
    if (ms->three_d) {
      PR(DUSTB_IPY, p) = x0[1] + dt*(vh[1] - (sbox ? q*om*xh[0] : 0.0));
      PR(DUSTB_IPZ, p) = x0[2] + dt*vh[2];
    } else {
      PR(DUSTB_IPY, p) = x0[1] + dt*vh[1];
    }
    PR(DUSTB_IPX1, p) = xh[0]; PR(DUSTB_IPY1, p) = xh[1];
    if (ms->three_d) PR(DUSTB_IPZ1, p) = xh[2];
    const double dv[3] = {dt*(ug[0] - vh[0])/PR(DUSTB_IPTS, p),
                          dt*(ug[1] - vh[1])/PR(DUSTB_IPTS, p),
                          dt*(ug[2] - vh[2])/PR(DUSTB_IPTS, p)};
    PR(DUSTB_IPRX, p) = dv[0]; PR(DUSTB_IPRY, p) = dv[1]; PR(DUSTB_IPRZ, p) = dv[2];
    if (!br) continue;
    cloud_deposit(c, &d, m, xf, code, c->f.dmom, 3, 0, 3, -PR(DUSTB_IPM, p), dv, 0, NULL);
  }
  free(gp);
  return err;
}

double oracle_pc2_apply_predictor(const dustb_ctx *c, double dt);
void oracle_pc2_midpoint(const dustb_ctx *c);
void oracle_pc2_commit(const dustb_ctx *c, double wpred);

/* one pc2 cycle of the clouds: the order of oracle_pc2_cycle with the clouds' predictor and
 * advance (their deposits in the owner cells: no deposit exchanges) */
unsigned oracle_cloud_pc2_cycle(const dustb_ctx *c, double dt, double *chi_out,
                                double *x3_removed) {
  unsigned err = 0;
  const int br = c->phys.back_reaction;
  oracle_register_copy(c);
  oracle_gas_rk_noflux(c, 1.0, 0.0);
  double chi = 0.0;
  if (br) {
    err |= oracle_cloud_pc2_predictor(c, dt, 1);
    chi = oracle_pc2_apply_predictor(c, dt);
  }
  oracle_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0);
  oracle_pc2_midpoint(c);
  oracle_gas_rk_noflux(c, 0.5, 0.5);
  err |= oracle_cloud_pc2_advance(c, dt);
  err |= oracle_route(c, x3_removed);
  if (br) oracle_pc2_commit(c, 0.5);
  oracle_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0);
  if (chi_out) *chi_out = chi;
  return err;
}

/* one imex2+ cycle of refinable clouds on a uniform mesh: the task order of oracle_imex_cycle
 * with the clouds' deposit (into the owners: no deposit exchange), their dc1 / dc2 sweeps
 * (with back-reaction), gather-kick and PMBR split */
unsigned oracle_cloud_imex_cycle(const dustb_ctx *c, double gamma, double dt, const double sh[2],
                                 double *x3_removed) {
  double gam0[3], gam1[3], beta[3], atw22;
  oracle_imex2p_coeffs(gamma, gam0, gam1, beta, &atw22);
  const double a_dt = gamma*dt;
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  double *gp = (double *)malloc((size_t)ms->nmb*d.n3*d.n2*d.n1*12*sizeof(double));
  unsigned err = 0;
  for (int stage = 1; stage <= 2; ++stage) {
    if (stage == 1) oracle_register_copy(c);
    oracle_gas_rk_noflux(c, gam0[stage - 1], gam1[stage - 1]);
    if (stage == 2 && c->phys.back_reaction) oracle_history_gas(c, atw22*dt);
    oracle_push_imex(c, gam0[stage - 1], gam1[stage - 1], beta[stage - 1]*dt,
                     (stage == 2) ? atw22*dt : 0.0);
    err |= oracle_route(c, x3_removed);
    const double s = sh[stage - 1];
    if (c->phys.back_reaction) err |= oracle_cloud_deposit_qp(c, a_dt, s);
    oracle_solve_ustar(c);
    if (c->phys.back_reaction && c->phys.drag_solver >= DUSTB_SOLVER_DC1) {
      int nsweeps = (c->phys.drag_solver == DUSTB_SOLVER_DC2) ? 2 : 1;
      for (int w = 0; w < nsweeps; ++w) err |= oracle_cloud_dc1_sweep(c, a_dt, s);
    }
    cloud_copy_exchange(c, c->f.ustar, 3, 1);
    oracle_gather_pack(c, c->f.ustar, gp);
    err |= oracle_cloud_gather_kick(c, a_dt, s, gp);
    if (c->phys.back_reaction) oracle_cloud_apply_pmbr(c, a_dt, s);
    cloud_copy_exchange(c, c->f.u0, c->f.nvar_gas, 0);
  }
  free(gp);
  return err;
}

/* ---- the cloud order index, DustGasDrag::UpdateCloudOrder, src/dust/dust_cloud_device.cpp:
 * 1992-2055: the keys of SortParticles sorted, the particle of each slot and its 64-bit tag
 * (TagFromWords, src/athena.hpp:85-88) ------------------------------------------------- */
static uint64_t tag_words(int lo, int hi) {
  return ((uint64_t)(uint32_t)hi << 32) | (uint64_t)(uint32_t)lo;
}

void oracle_cloud_order(const dustb_ctx *c, int *ord, uint64_t *tag) {
  const int *pi = c->part.pi; long long stride = c->part.stride;
  oracle_sort_order(c, ord, NULL);
  for (int k = 0; k < c->part.npart; ++k)
    tag[k] = tag_words(PI(DUSTB_PTAG, ord[k]), PI(DUSTB_PTAGH, ord[k]));
}

/* the check between rebuilds (:2001-2010): entries whose slot is out of range or holds
 * another tag */
int oracle_cloud_order_check(const dustb_ctx *c, const int *ord, const uint64_t *tag, int n) {
  const int *pi = c->part.pi; long long stride = c->part.stride;
  int bad = 0;
  for (int k = 0; k < n; ++k) {
    const int p = ord[k];
    if (p < 0 || p >= c->part.npart ||
        tag_words(PI(DUSTB_PTAG, p), PI(DUSTB_PTAGH, p)) != tag[k]) ++bad;
  }
  return bad;
}

/* ---- pc2 ------------------------------------------------------------------------------ */
/* DepositDrag pc2 predictor, src/dust/dust_pm.cpp:109-194 (qdep zeroed first) */
unsigned oracle_pc2_predictor(const dustb_ctx *c, double dt, int rate_dep) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  memset(c->f.qdep, 0, field_size(ms, 5)*sizeof(double));
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const double *uold = c->f.u1;
  const int clo = ms->three_d ? 0 : 1, chi = ms->three_d ? 2 : 1;
  unsigned err = 0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) reduction(| : err)
  for (int p = 0; p < c->part.npart; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    int ip, jp, kp; double wx[3], wy[3], wz[3];
    particle_weights(c, &d, m, PR(DUSTB_IPX, p), PR(DUSTB_IPY, p), PR(DUSTB_IPZ, p),
                     &ip, &jp, &kp, wx, wy, wz);
    if (!halo_ok(ms, &d, ip, jp, kp)) { err |= DUSTB_ERR_HALO; continue; }
    double ugx = 0.0, ugy = 0.0, ugz = 0.0;
    for (int cc = clo; cc <= chi; ++cc)
      for (int b = 0; b < 3; ++b) {
        double wcb = wz[cc]*wy[b];
        if (wcb == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
          double w = wcb*wx[a];
          int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
          double invrho = 1.0/A5(uold, nv, d, m, 0, kk, jj, ii);
          ugx += w*A5(uold, nv, d, m, 1, kk, jj, ii)*invrho;
          ugy += w*A5(uold, nv, d, m, 2, kk, jj, ii)*invrho;
          ugz += w*A5(uold, nv, d, m, 3, kk, jj, ii)*invrho;
        }
      }
    double vol = cell_volume(ms, m);
    double rate = PR(DUSTB_IPM, p)/(PR(DUSTB_IPTS, p)*vol);
    double gx = -dt*rate*(ugx - PR(DUSTB_IPVX, p));
    double gy = -dt*rate*(ugy - PR(DUSTB_IPVY, p));
    double gz = -dt*rate*(ugz - PR(DUSTB_IPVZ, p));
    for (int cc = clo; cc <= chi; ++cc)
      for (int b = 0; b < 3; ++b) {
        double wcb = wz[cc]*wy[b];
        if (wcb == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
          double w = wcb*wx[a];
          int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
          deposit_add(&A5(c->f.qdep, 5, d, m, 1, kk, jj, ii), w*gx);
          deposit_add(&A5(c->f.qdep, 5, d, m, 2, kk, jj, ii), w*gy);
          deposit_add(&A5(c->f.qdep, 5, d, m, 3, kk, jj, ii), w*gz);
          if (rate_dep) deposit_add(&A5(c->f.qdep, 5, d, m, 4, kk, jj, ii), w*rate);
        }
      }
  }
  return err;
}

/* GasImplicitSolve pc2 stage 1, src/dust/dust_pm.cpp:374-405, with UpdateStiffness's
 * maximum (dust_pm.cpp:288-300) returned as chi = dt*max(qdep4/rho) */
double oracle_pc2_apply_predictor(const dustb_ctx *c, double dt) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  double rate = 0.0;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i)
          rate = fmax(rate, A5(c->f.qdep, 5, d, m, 4, k, j, i)/A5(c->f.u0, nv, d, m, 0, k, j, i));
  const int damp = c->phys.pc2_feedback_damping;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i) {
          if (damp) {
            const double chi = dt*A5(c->f.qdep, 5, d, m, 4, k, j, i)/A5(c->f.u0, nv, d, m, 0, k, j, i);
            if (chi > 1.0) {
              const double s = 1.0/chi;
              for (int v = 1; v <= 3; ++v) A5(c->f.qdep, 5, d, m, v, k, j, i) *= s;
            }
          }
          for (int v = 1; v <= 3; ++v)
            A5(c->f.u0, nv, d, m, v, k, j, i) += A5(c->f.qdep, 5, d, m, v, k, j, i);
        }
  return dt*rate;
}

/* FirstTwoImpRK pc2 stage 2, src/dust/dust_push.cpp:37-61 (ghosts included) */
void oracle_pc2_midpoint(const dustb_ctx *c) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = 0; k < d.n3; ++k)
      for (int j = 0; j < d.n2; ++j)
        for (int i = 0; i < d.n1; ++i) {
          double inv = 1.0/(A5(c->f.u1, nv, d, m, 0, k, j, i) + A5(c->f.u0, nv, d, m, 0, k, j, i));
          for (int v = 0; v < 3; ++v)
            A5(c->f.ustar, 3, d, m, v, k, j, i) =
                (A5(c->f.u1, nv, d, m, 1 + v, k, j, i) + A5(c->f.u0, nv, d, m, 1 + v, k, j, i))*inv;
        }
}

/* ExplicitPush pc2 advance, src/dust/dust_push.cpp:99-247 (dmom zeroed first) */
unsigned oracle_pc2_advance(const dustb_ctx *c, double dt) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms);
  const int br = c->phys.back_reaction, three_d = ms->three_d;
  const int sbox = c->phys.shearing_box, strat = c->phys.stratified;
  const double q = c->phys.qshear, om = c->phys.omega0, aphi = c->phys.const_accel_phi;
  if (br) memset(c->f.dmom, 0, field_size(ms, 3)*sizeof(double));
  double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const int clo = three_d ? 0 : 1, chi = three_d ? 2 : 1;
  unsigned err = 0;
#pragma omp parallel for if (g_threads > 1) num_threads(g_threads) reduction(| : err)
  for (int p = 0; p < c->part.npart; ++p) {
    int m = PI(DUSTB_PGID, p) - ms->gids;
    double x0 = PR(DUSTB_IPX1, p), y0 = PR(DUSTB_IPY1, p), z0 = PR(DUSTB_IPZ1, p);
    double vx0 = PR(DUSTB_IPVX1, p), vy0 = PR(DUSTB_IPVY1, p), vz0 = PR(DUSTB_IPVZ1, p);
    double xh = x0 + 0.5*dt*vx0;
    double yh = y0 + 0.5*dt*(vy0 - ((sbox && three_d) ? q*om*x0 : 0.0));
    double zh = three_d ? z0 + 0.5*dt*vz0 : z0;
    double yg = yh + ((sbox && three_d) ? q*om*xh*0.5*dt : 0.0);
    int ip, jp, kp; double wx[3], wy[3], wz[3];
    particle_weights(c, &d, m, xh, yg, zh, &ip, &jp, &kp, wx, wy, wz);
    if (!halo_ok(ms, &d, ip, jp, kp)) { err |= DUSTB_ERR_HALO; continue; }
    double ugx = 0.0, ugy = 0.0, ugz = 0.0;
    for (int cc = clo; cc <= chi; ++cc)
      for (int b = 0; b < 3; ++b) {
        double wcb = wz[cc]*wy[b];
        if (wcb == 0.0) continue;
        for (int a = 0; a < 3; ++a) {
          double w = wcb*wx[a];
          int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
          ugx += w*A5(c->f.ustar, 3, d, m, 0, kk, jj, ii);
          ugy += w*A5(c->f.ustar, 3, d, m, 1, kk, jj, ii);
          ugz += w*A5(c->f.ustar, 3, d, m, 2, kk, jj, ii);
        }
      }
    double h = 0.5*dt;
    double lambda = h/PR(DUSTB_IPTS, p);
    double aa = 1.0 + lambda;
    double rx = vx0 + lambda*ugx, ry = vy0 + lambda*ugy, rz = vz0 + lambda*ugz;
    double vxh, vyh, vzh;
    if (sbox && three_d) {
      double cxy = 2.0*h*om, cyx = h*(2.0 - q)*om;
      double det = aa*aa + cxy*cyx;
      vxh = (aa*rx + cxy*ry)/det;
      vyh = (aa*ry - cyx*rx)/det;
      if (strat) rz -= h*SQR(om)*zh;
      vzh = rz/aa;
    } else if (sbox) {
      double cxz = 2.0*h*om, czx = h*(2.0 - q)*om;
      double det = aa*aa + cxz*czx;
      if (aphi != 0.0) rz += h*aphi;
      vxh = (aa*rx + cxz*rz)/det;
      vzh = (aa*rz - czx*rx)/det;
      vyh = ry/aa;
    } else {
      vxh = rx/aa; vyh = ry/aa; vzh = rz/aa;
    }
    PR(DUSTB_IPVX, p) = 2.0*vxh - vx0;
    PR(DUSTB_IPVY, p) = 2.0*vyh - vy0;
    PR(DUSTB_IPVZ, p) = 2.0*vzh - vz0;
    PR(DUSTB_IPX, p) = x0 + dt*vxh;
    PR(DUSTB_IPY, p) = y0 + dt*(vyh - ((sbox && three_d) ? q*om*xh : 0.0));
    if (three_d) PR(DUSTB_IPZ, p) = z0 + dt*vzh;
    PR(DUSTB_IPX1, p) = xh; PR(DUSTB_IPY1, p) = yh; PR(DUSTB_IPZ1, p) = zh;
    double dvx = dt*(ugx - vxh)/PR(DUSTB_IPTS, p);
    double dvy = dt*(ugy - vyh)/PR(DUSTB_IPTS, p);
    double dvz = dt*(ugz - vzh)/PR(DUSTB_IPTS, p);
    PR(DUSTB_IPRX, p) = dvx; PR(DUSTB_IPRY, p) = dvy; PR(DUSTB_IPRZ, p) = dvz;
    if (br) {
      double vol = cell_volume(ms, m);
      double fac = -PR(DUSTB_IPM, p)/vol;
      for (int cc = clo; cc <= chi; ++cc)
        for (int b = 0; b < 3; ++b) {
          double wcb = wz[cc]*wy[b]*fac;
          if (wcb == 0.0) continue;
          for (int a = 0; a < 3; ++a) {
            double w = wcb*wx[a];
            int kk = kp + cc - 1, jj = jp + b - 1, ii = ip + a - 1;
            deposit_add(&A5(c->f.dmom, 3, d, m, 0, kk, jj, ii), w*dvx);
            deposit_add(&A5(c->f.dmom, 3, d, m, 1, kk, jj, ii), w*dvy);
            deposit_add(&A5(c->f.dmom, 3, d, m, 2, kk, jj, ii), w*dvz);
          }
        }
    }
  }
  return err;
}

/* ApplyPMBR pc2 commit, src/dust/dust_pm.cpp:585-602 */
void oracle_pc2_commit(const dustb_ctx *c, double wpred) {
  const dustb_mesh *ms = &c->mesh; Ind d = indices(ms); int nv = c->f.nvar_gas;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = d.ks; k <= d.ke; ++k)
      for (int j = d.js; j <= d.je; ++j)
        for (int i = d.is; i <= d.ie; ++i)
          for (int v = 0; v < 3; ++v)
            A5(c->f.u0, nv, d, m, 1 + v, k, j, i) +=
                A5(c->f.dmom, 3, d, m, v, k, j, i) - wpred*A5(c->f.qdep, 5, d, m, 1 + v, k, j, i);
}

/* ---- cycle drivers: the task order of src/dust/dust_tasks.cpp:38-120 -------------------- */

/* imex2+ tableau, src/driver/driver.cpp:278-300 */
/* ---- ParticleHistory, src/dust/dust_science.cpp:391-482 (3-D point particles) ----------
 * row[0..6]: the particle sums, chunks of 4096 particles each summed in particle order, the
 * chunks summed in order (:398-418); row[7..11]: the densest active cell of the mass deposit
 * (DepositPointScienceFields, src/dust/dust_gravity_points.cpp:277-309: m/V times the deposit
 * weights, the ghost deposits summed into their owners) and its centre, the first cell in
 * (block, k, j, i) order among equal values (:428-441); row[12]: *chi (back-reaction) or -1;
 * row[13] -1, row[14..15] 0.  field: nmb cells of one variable (ghosts included), scratch. */
/* ---- point-particle fields for self-gravity and outputs, src/dust/dust_gravity_points.cpp ---
 * A 3-D point particle the transfers accept (:216-223, :282-287): a finite mass (gravity: also
 * >= 0), an owner block in the pack, a finite position, a stencil inside the padded block.
 * Massless particles contribute nothing. */
static int point_stencil(const dustb_ctx *c, const Ind *d, int p, int *m, int *ip, int *jp,
                         int *kp, double wx[3], double wy[3], double wz[3]) {
  const dustb_mesh *ms = &c->mesh;
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  *m = PI(DUSTB_PGID, p) - ms->gids;
  const double x = PR(DUSTB_IPX, p), y = PR(DUSTB_IPY, p), z = PR(DUSTB_IPZ, p);
  if (*m < 0 || *m >= ms->nmb || !isfinite(x) || !isfinite(y) || !isfinite(z)) return 0;
  particle_weights(c, d, *m, x, y, z, ip, jp, kp, wx, wy, wz);
  return *ip >= 1 && *ip < d->n1 - 1 && *jp >= 1 && *jp < d->n2 - 1 && *kp >= 1 &&
         *kp < d->n3 - 1;
}

/* DepositPointGravityDensity (:215-249, gravity = 1) and DepositPointScienceFields (:257-305):
 * the densities into a field with ghosts, the remap with the fold at physical x3 faces (the
 * transfers' plans, :176-178), the active cells copied out, the ghost cells zero */
static unsigned point_deposit(const dustb_ctx *c, double *out, int ncomp, int species,
                              int gravity) {
  const dustb_mesh *ms = &c->mesh; const Ind d = indices(ms);
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  const size_t nf = field_size(ms, ncomp);
  double *f = (double *)calloc(nf, sizeof(double));
  unsigned err = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    const double mass = PR(DUSTB_IPM, p);
    if (gravity) {
      if (!(mass >= 0.0) || !isfinite(mass)) { err |= DUSTB_ERR_POINT; continue; }
      if (mass == 0.0) continue;
    } else {
      if (mass == 0.0) continue;
      if (species >= 0 && PI(DUSTB_PSP, p) != species) continue;
      if (!isfinite(mass)) { err |= DUSTB_ERR_POINT; continue; }
    }
    int m, ip, jp, kp; double wx[3], wy[3], wz[3];
    if (!point_stencil(c, &d, p, &m, &ip, &jp, &kp, wx, wy, wz)) { err |= DUSTB_ERR_POINT; continue; }
    const double density = mass/(MB(m, DX1)*MB(m, DX2)*MB(m, DX3));
    const double v[3] = {PR(DUSTB_IPVX, p), PR(DUSTB_IPVY, p), PR(DUSTB_IPVZ, p)};
    for (int cc = 0; cc < 3; ++cc)
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
          const double w = density*wz[cc]*wy[b]*wx[a];
          if (w == 0.0) continue;
          A5(f, ncomp, d, m, 0, kp + cc - 1, jp + b - 1, ip + a - 1) += w;
          for (int q = 1; q < ncomp; ++q)
            A5(f, ncomp, d, m, q, kp + cc - 1, jp + b - 1, ip + a - 1) += w*v[q - 1];
        }
  }
  dustb_ctx g = *c;
  g.phys.x3_deposit_drop = 0;
  oracle_ghost_add(&g, f, ncomp);
  memset(out, 0, nf*sizeof(double));
  for (int m = 0; m < ms->nmb; ++m)
    for (int q = 0; q < ncomp; ++q)
      for (int k = d.ks; k <= d.ke; ++k)
        for (int j = d.js; j <= d.je; ++j)
          for (int i = d.is; i <= d.ie; ++i)
            A5(out, ncomp, d, m, q, k, j, i) = A5(f, ncomp, d, m, q, k, j, i);
  free(f);
  return err;
}

unsigned oracle_point_gravity_density(const dustb_ctx *c, double *owned) {
  return point_deposit(c, owned, 1, -1, 1);
}

unsigned oracle_point_science_fields(const dustb_ctx *c, double *out, int mass_only,
                                     int species) {
  return point_deposit(c, out, mass_only ? 1 : 4, species, 0);
}

/* The force field of GatherPointGravityAcceleration (:325-337): owned on the active cells, and
 * the transpose of the deposit remap (GatherMap, :121-160) for the ghost cells: every entry
 * (target active cell, source ghost cell, weight) of oracle_ghost_add's remap, with the fold at
 * physical x3 faces, adds weight * owned(target) into the source ghost cell. */
static void point_force_field(const dustb_ctx *c0, const double *owned, double *f) {
  dustb_ctx cg = *c0;
  cg.phys.x3_deposit_drop = 0;
  const dustb_ctx *c = &cg;
  const dustb_mesh *ms = &c->mesh; const Ind d = indices(ms);
  const int nvar = 3, ng1 = ms->ng - 1, ndir = 26;
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  memset(f, 0, field_size(ms, nvar)*sizeof(double));
  for (int m = 0; m < ms->nmb; ++m)
    for (int v = 0; v < nvar; ++v)
      for (int k = d.ks; k <= d.ke; ++k)
        for (int j = d.js; j <= d.je; ++j)
          for (int i = d.is; i <= d.ie; ++i)
            A5(f, nvar, d, m, v, k, j, i) = A5(owned, nvar, d, m, v, k, j, i);
  /* the same-level exchange: receiver m's strip facing direction o took the neighbour's ghost
   * cells at index - o nx */
  for (int m = 0; m < ms->nmb; ++m)
    for (int n = 0; n < ndir; ++n) {
      const int *o = kDirOrder[n];
      const int gid = ms->nghbr[(size_t)m*27 + (o[2] + 1)*9 + (o[1] + 1)*3 + (o[0] + 1)];
      if (gid < 0 || shear_crossing(c, m, o[0])) continue;
      const int src = gid - ms->gids;
      int lo[3], hi[3];
      const int s[3] = {d.is, d.js, d.ks}, e[3] = {d.ie, d.je, d.ke};
      for (int ax = 0; ax < 3; ++ax) {
        lo[ax] = (o[ax] > 0) ? (e[ax] - ng1) : s[ax];
        hi[ax] = (o[ax] < 0) ? (s[ax] + ng1) : e[ax];
      }
      for (int v = 0; v < nvar; ++v)
        for (int k = lo[2]; k <= hi[2]; ++k)
          for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i)
              A5(f, nvar, d, src, v, k - o[2]*nx[2], j - o[1]*nx[1], i - o[0]*nx[0]) +=
                  A5(owned, nvar, d, m, v, k, j, i);
    }
  /* the fold behind physical x3 faces */
  if (ms->x3bc != 0)
    for (int m = 0; m < ms->nmb; ++m)
      for (int side = 0; side < 2; ++side) {
        const int o3 = side ? 1 : -1;
        if (ms->nghbr[(size_t)m*27 + (o3 + 1)*9 + 1*3 + 1] >= 0) continue;
        for (int t = 0; t < ms->ng; ++t) {
          const int k = side ? d.ke - t : d.ks + t;
          const int kg = side ? d.ke + 1 + t : d.ks - 1 - t;
          for (int v = 0; v < nvar; ++v)
            for (int j = d.js; j <= d.je; ++j)
              for (int i = d.is; i <= d.ie; ++i) {
                const double val = A5(owned, nvar, d, m, v, k, j, i);
                A5(f, nvar, d, m, v, kg, j, i) += val;
                for (int n = 0; n < ndir; ++n) {
                  const int *o = kDirOrder[n];
                  if (o[2] != 0) continue;
                  if (o[0] > 0 && i < d.ie - ng1) continue;
                  if (o[0] < 0 && i > d.is + ng1) continue;
                  if (o[1] > 0 && j < d.je - ng1) continue;
                  if (o[1] < 0 && j > d.js + ng1) continue;
                  const int gid = ms->nghbr[(size_t)m*27 + 1*9 + (o[1] + 1)*3 + (o[0] + 1)];
                  if (gid < 0 || shear_crossing(c, m, o[0])) continue;
                  A5(f, nvar, d, gid - ms->gids, v, kg, j - o[1]*nx[1], i - o[0]*nx[0]) += val;
                }
              }
        }
      }
  /* the shear-periodic faces */
  if (!ms->shear_x1) return;
  for (int m = 0; m < ms->nmb; ++m) {
    if (!sb_faces(ms, m)) continue;
    for (int v = 0; v < nvar; ++v)
      for (int k = d.ks; k <= d.ke; ++k)
        for (int j = d.js; j <= d.je; ++j)
          for (int i = d.is; i <= d.ie; ++i)
            shear_remap_entries(c, &d, NULL, nvar, m, v, k, j, i, f,
                                A5(owned, nvar, d, m, v, k, j, i));
  }
}

void oracle_point_force_field(const dustb_ctx *c, const double *owned, double *f) {
  point_force_field(c, owned, f);
}

/* GatherPointGravityAcceleration (:316-369): acc[v * acc_stride + p] = the TSC weights of the
 * particle over the force field */
unsigned oracle_point_gravity_gather(const dustb_ctx *c, const double *owned, double *acc,
                                     long long acc_stride) {
  const dustb_mesh *ms = &c->mesh; const Ind d = indices(ms);
  const double *pr = c->part.pr; const int *pi = c->part.pi; long long stride = c->part.stride;
  (void)pi;
  double *f = (double *)malloc(field_size(ms, 3)*sizeof(double));
  point_force_field(c, owned, f);
  unsigned err = 0;
  for (int p = 0; p < c->part.npart; ++p) {
    double a[3] = {0.0, 0.0, 0.0};
    const double mass = PR(DUSTB_IPM, p);
    int m, ip, jp, kp; double wx[3], wy[3], wz[3];
    if (!(mass >= 0.0) || !isfinite(mass)) {
      err |= DUSTB_ERR_POINT;
    } else if (mass != 0.0) {
      if (!point_stencil(c, &d, p, &m, &ip, &jp, &kp, wx, wy, wz)) {
        err |= DUSTB_ERR_POINT;
      } else {
        for (int cc = 0; cc < 3; ++cc)
          for (int b = 0; b < 3; ++b)
            for (int q = 0; q < 3; ++q) {
              const double w = wz[cc]*wy[b]*wx[q];
              for (int v = 0; v < 3; ++v)
                a[v] += w*A5(f, 3, d, m, v, kp + cc - 1, jp + b - 1, ip + q - 1);
            }
        if (!isfinite(a[0]) || !isfinite(a[1]) || !isfinite(a[2])) err |= DUSTB_ERR_POINT;
      }
    }
    for (int v = 0; v < 3; ++v) acc[(size_t)v*acc_stride + p] = a[v];
  }
  free(f);
  return err;
}

unsigned oracle_phst(const dustb_ctx *c, const double *chi, double *field, double row[16]) {
  const dustb_mesh *ms = &c->mesh;
  const double *pr = c->part.pr;
  const int *pi = c->part.pi;
  const size_t stride = (size_t)c->part.stride;
  const int np = c->part.npart;
  const int zc = ms->three_d ? DUSTB_IPZ : DUSTB_IPY;
  double sums[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int c0 = 0; c0 < np; c0 += 4096) {
    double a[7] = {0, 0, 0, 0, 0, 0, 0};
    const int p1 = (c0 + 4096 < np) ? c0 + 4096 : np;
    for (int p = c0; p < p1; ++p) {
      const double m = PR(DUSTB_IPM, p);
      if (m == 0.0) continue;
      const double v1 = PR(DUSTB_IPVX, p), v2 = PR(DUSTB_IPVY, p), v3 = PR(DUSTB_IPVZ, p);
      const double z = PR(zc, p);
      a[0] += 1.0;
      a[1] += m;
      a[2] += m*v1; a[3] += m*v2; a[4] += m*v3;
      a[5] += 0.5*m*(v1*v1 + v2*v2 + v3*v3);
      a[6] += m*z*z;
    }
    for (int q = 0; q < 7; ++q) sums[q] += a[q];
  }
  for (int q = 0; q < 6; ++q) row[q] = sums[q];
  row[6] = (sums[1] > 0.0) ? sqrt(sums[6]/sums[1]) : 0.0;
  /* the mass deposit */
  const Ind d = indices(ms);
  memset(field, 0, field_size(ms, 1)*sizeof(double));
  unsigned err = 0;
  for (int p = 0; p < np; ++p) {
    const double mass = PR(DUSTB_IPM, p);
    if (mass == 0.0) continue;
    const int m = PI(DUSTB_PGID, p) - ms->gids;
    if (m < 0 || m >= ms->nmb) { err |= DUSTB_ERR_PGID; continue; }
    int ip, jp, kp; double wx[3], wy[3], wz[3];
    particle_weights(c, &d, m, PR(DUSTB_IPX, p), PR(DUSTB_IPY, p), PR(DUSTB_IPZ, p), &ip, &jp,
                     &kp, wx, wy, wz);
    if (!halo_ok(ms, &d, ip, jp, kp)) { err |= DUSTB_ERR_HALO; continue; }
    const double density = mass/cell_volume(ms, m);
    for (int cc = 0; cc < 3; ++cc)
      for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) {
          const double w = density*wz[cc]*wy[b]*wx[a];
          if (w == 0.0) continue;
          A5(field, 1, d, m, 0, kp + cc - 1, jp + b - 1, ip + a - 1) += w;
        }
  }
  oracle_ghost_add(c, field, 1);
  double best = 0.0;
  long long loc = -1;
  const long long ncell = (long long)ms->nx1*ms->nx2*ms->nx3;
  for (int m = 0; m < ms->nmb; ++m)
    for (int k = 0; k < ms->nx3; ++k)
      for (int j = 0; j < ms->nx2; ++j)
        for (int i = 0; i < ms->nx1; ++i) {
          const double v = A5(field, 1, d, m, 0, d.ks + k, d.js + j, d.is + i);
          if (v > best) { best = v; loc = ((long long)m*ncell + ((long long)k*ms->nx2 + j)*ms->nx1 + i); }
        }
  row[7] = best;
  row[8] = row[9] = row[10] = 0.0;
  row[11] = -1.0;
  if (loc >= 0) {
    const int m = (int)(loc/ncell);
    const long long r = loc % ncell;
    const int k = (int)(r/((long long)ms->nx1*ms->nx2)), j = (int)((r/ms->nx1) % ms->nx2), i = (int)(r % ms->nx1);
    row[8] = MB(m, X1MIN) + (i + 0.5)*MB(m, DX1);
    row[9] = MB(m, X2MIN) + (j + 0.5)*MB(m, DX2);
    row[10] = ms->three_d ? MB(m, X3MIN) + (k + 0.5)*MB(m, DX3) : 0.0;
    row[11] = 0.0;
  }
  row[12] = (c->phys.back_reaction && chi) ? *chi : -1.0;
  row[13] = -1.0;
  row[14] = 0.0;
  row[15] = 0.0;
  return err;
}

void oracle_imex2p_coeffs(double gamma, double gam0[3], double gam1[3], double beta[3],
                          double *atw22) {
  gam0[0] = 1.0; gam1[0] = 0.0; beta[0] = gamma;
  gam0[1] = (2.0*gamma - 1.0)/(2.0*gamma*gamma);
  gam1[1] = (1.0 - (2.0*gamma - 1.0)/(2.0*gamma*gamma));
  beta[1] = 1.0/(2.0*gamma);
  gam0[2] = 1.0; gam1[2] = 0.0; beta[2] = 0.0;
  *atw22 = (1.0 - 2.0*gamma*gamma)/2.0/gamma;
}

/* one imex2+ cycle; sh[s] is ImplicitShearShift of working stage s+1 */
unsigned oracle_imex_cycle(const dustb_ctx *c, double gamma, double dt, const double sh[2],
                           double *x3_removed) {
  double gam0[3], gam1[3], beta[3], atw22;
  oracle_imex2p_coeffs(gamma, gam0, gam1, beta, &atw22);
  const double a_dt = gamma*dt;
  unsigned err = 0;
  for (int stage = 1; stage <= 2; ++stage) {
    if (stage == 1) oracle_register_copy(c);
    /* gas chain: RKUpdate stand-in, then the drag history term */
    oracle_gas_rk_noflux(c, gam0[stage - 1], gam1[stage - 1]);
    if (stage == 2 && c->phys.back_reaction) oracle_history_gas(c, atw22*dt);
    /* particle chain */
    oracle_push_imex(c, gam0[stage - 1], gam1[stage - 1], beta[stage - 1]*dt,
                     (stage == 2) ? atw22*dt : 0.0);
    err |= oracle_route(c, x3_removed);
    const double s = sh[stage - 1];
    if (c->phys.back_reaction) {
      err |= oracle_deposit_qp(c, a_dt, s);
      oracle_ghost_add(c, c->f.qdep, 5);
    }
    oracle_solve_ustar(c);
    if (c->phys.back_reaction && c->phys.drag_solver >= DUSTB_SOLVER_DC1) {
      int nsweeps = (c->phys.drag_solver == DUSTB_SOLVER_DC2) ? 2 : 1;
      for (int w = 0; w < nsweeps; ++w) err |= oracle_dc1_sweep(c, a_dt, s);
    }
    oracle_ghost_copy(c, c->f.ustar, 3, 1);
    err |= oracle_gather_kick_pmbr(c, a_dt, s);
    if (c->phys.back_reaction) {
      oracle_ghost_add(c, c->f.dmom, 3);
      oracle_apply_pmbr(c, a_dt);
    }
    /* gas tail: the ghost exchange of the conserved state */
    oracle_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0);
  }
  return err;
}

/* one pc2 cycle (integrator rk2: gam0 = {1, 1/2}, gam1 = {0, 1/2}) */
unsigned oracle_pc2_cycle(const dustb_ctx *c, double dt, double *chi_out, double *x3_removed) {
  unsigned err = 0;
  const int br = c->phys.back_reaction;
  /* stage 1 */
  oracle_register_copy(c);
  oracle_gas_rk_noflux(c, 1.0, 0.0);
  double chi = 0.0;
  if (br) {
    err |= oracle_pc2_predictor(c, dt, 1);
    oracle_ghost_add(c, c->f.qdep, 5);
    chi = oracle_pc2_apply_predictor(c, dt);
  }
  oracle_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0);
  /* stage 2 */
  oracle_pc2_midpoint(c);
  oracle_gas_rk_noflux(c, 0.5, 0.5);
  err |= oracle_pc2_advance(c, dt);
  err |= oracle_route(c, x3_removed);
  if (br) {
    oracle_ghost_add(c, c->f.dmom, 3);
    oracle_pc2_commit(c, 0.5);
  }
  oracle_ghost_copy(c, c->f.u0, c->f.nvar_gas, 0);
  if (chi_out) *chi_out = chi;
  return err;
}

/* ---- the general deposit remap of a refined 3-D mesh, by brute force ------------------------
 * The static part of DepRemapPlan (src/bvals/bvals_dep_general.cpp:1-35, :62-160, :383-545):
 * every ghost cell of every block is given to the active cells it overlaps, weight = overlap
 * volume / target cell volume in finest-level units, and per target cell its sources ordered by
 * (source gid, source cell).  The reference intersects intervals direction by direction over a
 * target's neighbour list; this restatement instead cuts each ghost cell into finest-level unit
 * cubes and looks each cube's owner up in a finest-level ownership grid, counting the cubes a
 * (target cell, source cell) pair shares, which checks the neighbour-based build independently.
 * geo: nx1..3, ng, nmb_root1..3, root_level, max_level, x3mode (0 periodic, 1 fold, 2 drop);
 * lloc: level, lx1, lx2, lx3 per block.  Returns 0, -1 for invalid input, -3 for small capacities
 * (the counts are written either way). */
typedef struct { int tflat, sgid, scell; int cnt; } DepEnt;

static int cmp_depent(const void *a, const void *b) {
  const DepEnt *x = (const DepEnt *)a, *y = (const DepEnt *)b;
  if (x->tflat != y->tflat) return x->tflat < y->tflat ? -1 : 1;
  if (x->sgid != y->sgid) return x->sgid < y->sgid ? -1 : 1;
  if (x->scell != y->scell) return x->scell < y->scell ? -1 : 1;
  return 0;
}

int oracle_dep_plan(const int *geo, int nmb, const int *lloc, int *counts, int *seg_tgt,
                    int *seg_ptr, int *ent_src, double *ent_w, long long cap_seg,
                    long long cap_ent) {
  const int nx[3] = {geo[0], geo[1], geo[2]}, ng = geo[3];
  const int root = geo[7], R = geo[8], x3mode = geo[9];
  const int nc[3] = {nx[0] + 2*ng, nx[1] + 2*ng, nx[2] + 2*ng};
  const int ncell = nc[0]*nc[1]*nc[2];
  long long N[3];
  for (int d = 0; d < 3; ++d) N[d] = (long long)geo[4 + d]*nx[d]*(1LL << (R - root));
  const long long nunit = N[0]*N[1]*N[2];
  if (nunit <= 0 || nunit > (1LL << 28)) return -1;
  int *own = (int *)malloc((size_t)nunit*sizeof(int));
  for (long long u = 0; u < nunit; ++u) own[u] = -1;
  for (int m = 0; m < nmb; ++m) {
    const long long sc = 1LL << (R - lloc[4*m]);
    long long lo[3];
    for (int d = 0; d < 3; ++d) lo[d] = (long long)lloc[4*m + 1 + d]*nx[d]*sc;
    for (long long z = lo[2]; z < lo[2] + nx[2]*sc; ++z)
      for (long long y = lo[1]; y < lo[1] + nx[1]*sc; ++y)
        for (long long x = lo[0]; x < lo[0] + nx[0]*sc; ++x) own[(z*N[1] + y)*N[0] + x] = m;
  }
  size_t cap = 1 << 20, n = 0;
  DepEnt *e = (DepEnt *)malloc(cap*sizeof(DepEnt));
  int rc = 0;
  for (int m = 0; m < nmb && rc == 0; ++m) {
    const long long sc = 1LL << (R - lloc[4*m]);
    long long lo[3];
    for (int d = 0; d < 3; ++d) lo[d] = (long long)lloc[4*m + 1 + d]*nx[d]*sc;
    for (int k = 0; k < nc[2]; ++k)
      for (int j = 0; j < nc[1]; ++j)
        for (int i = 0; i < nc[0]; ++i) {
          if (i >= ng && i < nc[0] - ng && j >= ng && j < nc[1] - ng && k >= ng && k < nc[2] - ng)
            continue;
          const int scell = (k*nc[1] + j)*nc[0] + i;
          const long long a0[3] = {lo[0] + (i - ng)*sc, lo[1] + (j - ng)*sc, lo[2] + (k - ng)*sc};
          for (long long dz = 0; dz < sc; ++dz)
            for (long long dy = 0; dy < sc; ++dy)
              for (long long dx = 0; dx < sc; ++dx) {
                long long u[3] = {a0[0] + dx, a0[1] + dy, a0[2] + dz};
                int drop = 0;
                for (int d = 0; d < 3; ++d) {
                  if (u[d] >= 0 && u[d] < N[d]) continue;
                  if (d == 2 && x3mode != 0) {
                    if (x3mode == 2) { drop = 1; break; }
                    u[2] = (u[2] < 0) ? -u[2] - 1 : 2*N[2] - 1 - u[2];   /* mirror */
                  } else {
                    u[d] = (u[d] < 0) ? u[d] + N[d] : u[d] - N[d];
                  }
                }
                if (drop) continue;
                const int t = own[(u[2]*N[1] + u[1])*N[0] + u[0]];
                if (t < 0) { rc = -1; continue; }
                const long long tsc = 1LL << (R - lloc[4*t]);
                int tc[3];
                for (int d = 0; d < 3; ++d)
                  tc[d] = (int)((u[d] - (long long)lloc[4*t + 1 + d]*nx[d]*tsc)/tsc) + ng;
                if (n == cap) { cap *= 2; e = (DepEnt *)realloc(e, cap*sizeof(DepEnt)); }
                e[n].tflat = t*ncell + (tc[2]*nc[1] + tc[1])*nc[0] + tc[0];
                e[n].sgid = m; e[n].scell = scell; e[n].cnt = 1;
                ++n;
              }
        }
  }
  free(own);
  if (rc) { free(e); return rc; }
  qsort(e, n, sizeof(DepEnt), cmp_depent);
  /* merge the unit cubes of each (target cell, source cell) pair */
  size_t ne = 0;
  for (size_t q = 0; q < n; ++q) {
    if (ne > 0 && cmp_depent(&e[ne - 1], &e[q]) == 0) { e[ne - 1].cnt += 1; continue; }
    e[ne++] = e[q];
  }
  long long nseg = 0;
  for (size_t q = 0; q < ne; ++q) if (q == 0 || e[q].tflat != e[q - 1].tflat) ++nseg;
  counts[0] = (int)nseg; counts[1] = (int)ne; counts[2] = 0;
  if (seg_tgt && seg_ptr && ent_src && ent_w) {
    if (cap_seg < nseg || cap_ent < (long long)ne) { free(e); return -3; }
    long long s = 0;
    for (size_t q = 0; q < ne; ++q) {
      if (q == 0 || e[q].tflat != e[q - 1].tflat) { seg_tgt[s] = e[q].tflat; seg_ptr[s] = (int)q; ++s; }
      const int t = e[q].tflat/ncell;
      const double tsc = (double)(1LL << (R - lloc[4*t]));
      ent_src[q] = e[q].sgid*ncell + e[q].scell;
      ent_w[q] = (double)e[q].cnt/(tsc*tsc*tsc);
    }
    seg_ptr[nseg] = (int)ne;
  }
  free(e);
  return 0;
}

/* GeneralApply (src/bvals/bvals_dep_general.cpp:1135-1175): per target cell and variable the
 * weighted sum of its sources in list order, added once; a is (nmb, nvar, n3, n2, n1) with
 * ncell = n3 n2 n1 cells per block and variable. */
void oracle_dep_apply(int nseg, const int *seg_tgt, const int *seg_ptr, const int *ent_src,
                      const double *ent_w, double *a, int nvar, int ncell) {
  for (int s = 0; s < nseg; ++s) {
    const int tm = seg_tgt[s]/ncell, tc = seg_tgt[s] - tm*ncell;
    for (int v = 0; v < nvar; ++v) {
      double sum = 0.0;
      for (int q = seg_ptr[s]; q < seg_ptr[s + 1]; ++q) {
        const int sm = ent_src[q]/ncell, sc = ent_src[q] - sm*ncell;
        sum += ent_w[q]*a[((size_t)sm*nvar + v)*ncell + sc];
      }
      a[((size_t)tm*nvar + v)*ncell + tc] += sum;
    }
  }
}

/* ---- the copy exchange of a cell-centred field on a refined 3-D mesh ------------------------
 * AthenaK's multilevel cell-centred boundary values as the u* exchange uses them
 * (src/dust/dust_tasks.cpp:262-442): RestrictCC (src/mesh/mesh_refinement.cpp:1829-1880),
 * PackAndSendCC / RecvAndUnpackCC with the boxes of InitSendIndices / InitRecvIndices
 * (src/bvals/bvals_cc.cpp:53-460, src/bvals/buffs_cc.cpp:28-410), FillCoarseInBndryCC and
 * ProlongateCC with ProlongCC's min-mod slopes (src/bvals/prolongation.cpp:29-230,
 * src/mesh/prolongation.hpp:21-80).  The exchange runs as the reference's does, sender by
 * sender: every block packs the box of each slot and it lands in the receiver's buffer of the
 * slot the neighbour table names as its destination (MeshBlock::SetNeighbors' dest,
 * src/mesh/meshblock.cpp:142-420).  ca: nmb x nvar x (nx/2 + 2 ng)^3 scratch (cleared). */
static int nbr_index(int ix, int iy, int iz, int n1, int n2) {
  const int ax = ix < 0 ? -ix : ix, ay = iy < 0 ? -iy : iy;
  if (iz == 0) {
    if (ix*iy == 0) return ax*2*(ix + 1) + ay*2*(iy + 5) + n1 + 2*n2;
    return 16 + (ix + 1) + 2*(iy + 1) + n1;
  }
  if (ix*iy == 0) return 24 + ax*(ix + 9) + ay*(iy + 17) + 2*(iz + 1) + n1 + 2*n2;
  return 48 + (ix + 1)/2 + (iy + 1) + 2*(iz + 1);
}

typedef struct { int lo[3], hi[3]; } MlBox;
typedef struct { int nx[3], cnx[3], ng, is[3], ie[3], cis[3], cie[3], n[3], cn[3]; } MlGeo;

static void ml_slots(int tab[56][5]) {
  int s;
#define PUT(ix, iy, iz, a, b) do { s = nbr_index(ix, iy, iz, a, b); tab[s][0] = ix; \
    tab[s][1] = iy; tab[s][2] = iz; tab[s][3] = a; tab[s][4] = b; } while (0)
  for (int n = -1; n <= 1; n += 2) for (int fz = 0; fz < 2; ++fz) for (int fy = 0; fy < 2; ++fy) PUT(n, 0, 0, fy, fz);
  for (int m = -1; m <= 1; m += 2) for (int fz = 0; fz < 2; ++fz) for (int fx = 0; fx < 2; ++fx) PUT(0, m, 0, fx, fz);
  for (int m = -1; m <= 1; m += 2) for (int n = -1; n <= 1; n += 2) for (int fz = 0; fz < 2; ++fz) PUT(n, m, 0, fz, 0);
  for (int l = -1; l <= 1; l += 2) for (int fy = 0; fy < 2; ++fy) for (int fx = 0; fx < 2; ++fx) PUT(0, 0, l, fx, fy);
  for (int l = -1; l <= 1; l += 2) for (int n = -1; n <= 1; n += 2) for (int fy = 0; fy < 2; ++fy) PUT(n, 0, l, fy, 0);
  for (int l = -1; l <= 1; l += 2) for (int m = -1; m <= 1; m += 2) for (int fx = 0; fx < 2; ++fx) PUT(0, m, l, fx, 0);
  for (int l = -1; l <= 1; l += 2) for (int m = -1; m <= 1; m += 2) for (int n = -1; n <= 1; n += 2) PUT(n, m, l, 0, 0);
#undef PUT
}

/* InitSendIndices (3-D): kind 0 isame, 1 icoar (to a coarser neighbour), 2 ifine (to a finer) */
static MlBox ml_send(const MlGeo *g, const int *t, int kind) {
  MlBox b;
  const int ox1 = t[0], ox2 = t[1], ox3 = t[2], f1 = t[3], f2 = t[4], ng1 = g->ng - 1;
  const int o[3] = {ox1, ox2, ox3};
  for (int d = 0; d < 3; ++d) {
    const int s = (kind == 1) ? g->cis[d] : g->is[d], e = (kind == 1) ? g->cie[d] : g->ie[d];
    b.lo[d] = (o[d] > 0) ? (e - ng1) : s;
    b.hi[d] = (o[d] < 0) ? (s + ng1) : e;
  }
  if (kind == 2) {
    if (ox1 == 0) { if (f1 == 1) b.lo[0] += g->cnx[0] - g->ng; else b.hi[0] -= g->cnx[0] - g->ng; }
    if (ox2 == 0) {
      const int f = (ox1 != 0) ? f1 : f2;
      if (f == 1) b.lo[1] += g->cnx[1] - g->ng; else b.hi[1] -= g->cnx[1] - g->ng;
    }
    if (ox3 == 0) {
      const int f = (ox1 != 0 && ox2 != 0) ? f1 : f2;
      if (f == 1) b.lo[2] += g->cnx[2] - g->ng; else b.hi[2] -= g->cnx[2] - g->ng;
    }
  }
  return b;
}

/* InitRecvIndices (3-D): kind 0 isame, 1 icoar (from a coarser neighbour, into the coarse
 * array), 2 ifine (from a finer neighbour), 3 iprol (coarse cells to prolongate) */
static MlBox ml_recv(const MlGeo *g, const int *t, int kind) {
  MlBox b;
  const int o[3] = {t[0], t[1], t[2]}, f1 = t[3], f2 = t[4];
  const int w = (kind == 3) ? g->ng/2 : g->ng;
  for (int d = 0; d < 3; ++d) {
    const int coarse = (kind == 1 || kind == 3);
    const int s = coarse ? g->cis[d] : g->is[d], e = coarse ? g->cie[d] : g->ie[d];
    if (o[d] > 0) { b.lo[d] = e + 1; b.hi[d] = e + w; continue; }
    if (o[d] < 0) { b.lo[d] = s - w; b.hi[d] = s - 1; continue; }
    b.lo[d] = s; b.hi[d] = e;
    const int f = (d == 0) ? f1 : ((d == 1) ? ((o[0] != 0) ? f1 : f2)
                                            : ((o[0] != 0 && o[1] != 0) ? f1 : f2));
    if (kind == 1 || kind == 3) { if (f == 0) b.hi[d] += w; else b.lo[d] -= w; }
    else if (kind == 2) { if (f == 1) b.lo[d] += g->cnx[d]; else b.hi[d] -= g->cnx[d]; }
  }
  return b;
}

#define ML_F(m, v, k, j, i) a[((((size_t)(m)*nvar + (v))*g.n[2] + (k))*g.n[1] + (j))*g.n[0] + (i)]
#define ML_C(m, v, k, j, i) ca[((((size_t)(m)*nvar + (v))*g.cn[2] + (k))*g.cn[1] + (j))*g.cn[0] + (i)]

void oracle_ghost_copy_ml(const dustb_ctx *c, double *a, int nvar, double *ca) {
  const dustb_mesh *ms = &c->mesh;
  MlGeo g;
  const int nx[3] = {ms->nx1, ms->nx2, ms->nx3};
  g.ng = ms->ng;
  for (int d = 0; d < 3; ++d) {
    g.nx[d] = nx[d]; g.cnx[d] = nx[d]/2; g.is[d] = ms->ng; g.ie[d] = ms->ng + nx[d] - 1;
    g.cis[d] = ms->ng; g.cie[d] = ms->ng + nx[d]/2 - 1;
    g.n[d] = nx[d] + 2*ms->ng; g.cn[d] = nx[d]/2 + 2*ms->ng;
  }
  int tab[56][5];
  ml_slots(tab);
  const int nmb = ms->nmb;
  memset(ca, 0, (size_t)nmb*nvar*g.cn[0]*g.cn[1]*g.cn[2]*sizeof(double));
  /* RestrictCC */
  for (int m = 0; m < nmb; ++m)
    for (int v = 0; v < nvar; ++v)
      for (int k = g.cis[2]; k <= g.cie[2]; ++k)
        for (int j = g.cis[1]; j <= g.cie[1]; ++j)
          for (int i = g.cis[0]; i <= g.cie[0]; ++i) {
            const int fi = (i - g.cis[0])*2 + g.is[0], fj = (j - g.cis[1])*2 + g.is[1];
            const int fk = (k - g.cis[2])*2 + g.is[2];
            ML_C(m, v, k, j, i) = 0.125*(ML_F(m, v, fk, fj, fi) + ML_F(m, v, fk, fj, fi + 1)
                + ML_F(m, v, fk, fj + 1, fi) + ML_F(m, v, fk, fj + 1, fi + 1)
                + ML_F(m, v, fk + 1, fj, fi) + ML_F(m, v, fk + 1, fj, fi + 1)
                + ML_F(m, v, fk + 1, fj + 1, fi) + ML_F(m, v, fk + 1, fj + 1, fi + 1));
          }
  /* the exchange, sender by sender (every block's active or coarse cells are read, only
   * ghost cells are written, so the order does not matter) */
  for (int s = 0; s < nmb; ++s) {
    const int lev_s = ms->mb_lev[s];
    int myf[3];
    for (int d = 0; d < 3; ++d) {
      const double lo = (d == 0) ? ms->x1min : ((d == 1) ? ms->x2min : ms->x3min);
      const double l = MB(s, X1MAX + d) - MB(s, X1MIN + d);
      myf[d] = ((int)floor((MB(s, X1MIN + d) - lo)/l + 0.5)) & 1;
    }
    for (int n = 0; n < 56; ++n) {
      const int gr = ms->nghbr_ml[(size_t)s*56 + n];
      if (gr < 0) continue;
      const int r = gr - ms->gids;
      const int lev_r = ms->mb_lev[r];
      const int *t = tab[n];
      const int kind = (lev_r < lev_s) ? 1 : ((lev_r == lev_s) ? 0 : 2);
      const MlBox sb = ml_send(&g, t, kind);
      /* the receiver's slot pointing back (SetNeighbors' dest) */
      const int nd = abs(t[0]) + abs(t[1]) + abs(t[2]);
      int dn;
      if (lev_r == lev_s || nd == 3) dn = nbr_index(-t[0], -t[1], -t[2], 0, 0);
      else if (lev_r > lev_s) dn = nbr_index(-t[0], -t[1], -t[2], t[3], nd == 1 ? t[4] : 0);
      else if (nd == 1) {
        if (t[0] != 0) dn = nbr_index(-t[0], 0, 0, myf[1], myf[2]);
        else if (t[1] != 0) dn = nbr_index(0, -t[1], 0, myf[0], myf[2]);
        else dn = nbr_index(0, 0, -t[2], myf[0], myf[1]);
      } else {
        const int fd = (t[0] == 0) ? 0 : ((t[1] == 0) ? 1 : 2);
        dn = nbr_index(-t[0], -t[1], -t[2], myf[fd], 0);
      }
      /* the receiver's box for the sender's level */
      const int rkind = (lev_s < lev_r) ? 1 : ((lev_s == lev_r) ? 0 : 2);
      const MlBox rb = ml_recv(&g, tab[dn], rkind);
      const int ni = sb.hi[0] - sb.lo[0] + 1, nj = sb.hi[1] - sb.lo[1] + 1;
      const int nk = sb.hi[2] - sb.lo[2] + 1;
      for (int v = 0; v < nvar; ++v)
        for (int dk = 0; dk < nk; ++dk)
          for (int dj = 0; dj < nj; ++dj)
            for (int di = 0; di < ni; ++di) {
              const double val = (kind == 1) ? ML_C(s, v, sb.lo[2] + dk, sb.lo[1] + dj, sb.lo[0] + di)
                                             : ML_F(s, v, sb.lo[2] + dk, sb.lo[1] + dj, sb.lo[0] + di);
              if (rkind == 1) ML_C(r, v, rb.lo[2] + dk, rb.lo[1] + dj, rb.lo[0] + di) = val;
              else ML_F(r, v, rb.lo[2] + dk, rb.lo[1] + dj, rb.lo[0] + di) = val;
            }
    }
  }
  /* FillCoarseInBndryCC: the coarse ghost cells next to same-level neighbours */
  for (int m = 0; m < nmb; ++m)
    for (int n = 0; n < 56; ++n) {
      const int gs = ms->nghbr_ml[(size_t)m*56 + n];
      if (gs < 0 || ms->mb_lev[gs - ms->gids] != ms->mb_lev[m]) continue;
      const MlBox fb = ml_recv(&g, tab[n], 0);
      for (int v = 0; v < nvar; ++v)
        for (int k = (fb.lo[2] + g.cis[2])/2; k <= (fb.hi[2] + g.cis[2])/2; ++k)
          for (int j = (fb.lo[1] + g.cis[1])/2; j <= (fb.hi[1] + g.cis[1])/2; ++j)
            for (int i = (fb.lo[0] + g.cis[0])/2; i <= (fb.hi[0] + g.cis[0])/2; ++i) {
              const int fi = (i - g.cis[0])*2 + g.is[0], fj = (j - g.cis[1])*2 + g.is[1];
              const int fk = (k - g.cis[2])*2 + g.is[2];
              ML_C(m, v, k, j, i) = 0.125*(ML_F(m, v, fk, fj, fi) + ML_F(m, v, fk, fj, fi + 1)
                  + ML_F(m, v, fk, fj + 1, fi) + ML_F(m, v, fk, fj + 1, fi + 1)
                  + ML_F(m, v, fk + 1, fj, fi) + ML_F(m, v, fk + 1, fj, fi + 1)
                  + ML_F(m, v, fk + 1, fj + 1, fi) + ML_F(m, v, fk + 1, fj + 1, fi + 1));
            }
    }
  /* ProlongateCC: the fine ghost cells next to coarser neighbours */
  for (int m = 0; m < nmb; ++m)
    for (int n = 0; n < 56; ++n) {
      const int gs = ms->nghbr_ml[(size_t)m*56 + n];
      if (gs < 0 || ms->mb_lev[gs - ms->gids] >= ms->mb_lev[m]) continue;
      const MlBox pb = ml_recv(&g, tab[n], 3);
      for (int v = 0; v < nvar; ++v)
        for (int k = pb.lo[2]; k <= pb.hi[2]; ++k)
          for (int j = pb.lo[1]; j <= pb.hi[1]; ++j)
            for (int i = pb.lo[0]; i <= pb.hi[0]; ++i) {
#define SLOPE(dl, dr) (0.125*((((dl) < 0.0) ? -1.0 : 1.0) + (((dr) < 0.0) ? -1.0 : 1.0))*fmin(fabs(dl), fabs(dr)))
              const double cc = ML_C(m, v, k, j, i);
              const double d1 = SLOPE(cc - ML_C(m, v, k, j, i - 1), ML_C(m, v, k, j, i + 1) - cc);
              const double d2 = SLOPE(cc - ML_C(m, v, k, j - 1, i), ML_C(m, v, k, j + 1, i) - cc);
              const double d3 = SLOPE(cc - ML_C(m, v, k - 1, j, i), ML_C(m, v, k + 1, j, i) - cc);
#undef SLOPE
              const int fi = (i - g.cis[0])*2 + g.is[0], fj = (j - g.cis[1])*2 + g.is[1];
              const int fk = (k - g.cis[2])*2 + g.is[2];
              ML_F(m, v, fk, fj, fi) = cc - d1 - d2 - d3;
              ML_F(m, v, fk, fj, fi + 1) = cc + d1 - d2 - d3;
              ML_F(m, v, fk, fj + 1, fi) = cc - d1 + d2 - d3;
              ML_F(m, v, fk, fj + 1, fi + 1) = cc + d1 + d2 - d3;
              ML_F(m, v, fk + 1, fj, fi) = cc - d1 - d2 + d3;
              ML_F(m, v, fk + 1, fj, fi + 1) = cc + d1 - d2 + d3;
              ML_F(m, v, fk + 1, fj + 1, fi) = cc - d1 + d2 + d3;
              ML_F(m, v, fk + 1, fj + 1, fi + 1) = cc + d1 + d2 + d3;
            }
    }
}
#undef ML_F
#undef ML_C
