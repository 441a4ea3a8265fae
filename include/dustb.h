/*
 * dustb.h -- C ABI of the B200 dust particle-drag step.
 *
 * The entry points replace the dust task functions of AthenaK's DustGasDrag one for one
 * (reference: src/dust/dust_pm.cpp, dust_push.cpp, dust_solver.cpp, dust_newdt.cpp,
 * src/bvals/bvals_part.cpp, bvals_dep.cpp, dust_cloud_device.cpp).  Every pointer inside
 * dustb_ctx is a DEVICE pointer to an array the host code already owns, in the host code's
 * own layout:
 *
 *   particles  pr  = prtcl_rdata (17 x stride doubles, row r at pr + r*stride)
 *              pi  = prtcl_idata ( 5 x stride int32)     (src/particles/particles.cpp:96-113)
 *   mesh       u0, u1, qdep, ustar, dmom, resid, work:
 *              (nmb, nvar, n3, n2, n1) row-major doubles, n = nx + 2 ng per active direction
 *              (src/hydro/hydro.cpp:125, src/dust/dust.cpp:1160-1169)
 *   mb_size    nmb x 9 doubles {x1min,x2min,x3min,x1max,x2max,x3max,dx1,dx2,dx3}
 *              (RegionSize, src/mesh/mesh.hpp:25-29)
 *   nghbr      nmb x 27 int: gid of the same-level neighbour in direction (ox1,ox2,ox3),
 *              index (ox3+1)*9 + (ox2+1)*3 + (ox1+1), -1 where there is none
 *              (the first sub-slot NeighborIndex(ox1,ox2,ox3,0,0) of pmb->nghbr,
 *              src/mesh/nghbr_index.hpp:29)
 *
 * Every call takes the CUDA stream the host code runs on (Kokkos' default execution space
 * stream) as an opaque pointer, queues its kernels there and returns without waiting.
 * Return value: 0 on success, < 0 for an argument or launch error (DUSTB_E*).  Kernels
 * never trap: a violated invariant ORs a DUSTB_ERR_* bit into *ctx->err (device uint32) and
 * the offending particle is skipped, where the reference calls Kokkos::abort.
 *
 * No entry point allocates memory: scratch is passed by the caller (dustb_*_bytes).  The one
 * exception is dustb_cell_index_static, whose scratch is a fixed device array of the library
 * (DUSTB_STATIC_SCRATCH_BYTES on every GPU that loads it); its calls must not overlap on the
 * GPU.
 */
#ifndef DUSTB_H_
#define DUSTB_H_

#ifdef __cplusplus
extern "C" {
#endif

/* particle rows (src/athena.hpp:77-80) */
enum {
  DUSTB_IPX = 0, DUSTB_IPVX = 1, DUSTB_IPY = 2, DUSTB_IPVY = 3, DUSTB_IPZ = 4, DUSTB_IPVZ = 5,
  DUSTB_IPX1 = 6, DUSTB_IPVX1 = 7, DUSTB_IPY1 = 8, DUSTB_IPVY1 = 9, DUSTB_IPZ1 = 10,
  DUSTB_IPVZ1 = 11, DUSTB_IPRX = 12, DUSTB_IPRY = 13, DUSTB_IPRZ = 14, DUSTB_IPTS = 15,
  DUSTB_IPM = 16, DUSTB_NREAL = 17
};
enum { DUSTB_PGID = 0, DUSTB_PTAG = 1, DUSTB_PSP = 2, DUSTB_PLEV = 3, DUSTB_PTAGH = 4,
       DUSTB_NINT = 5 };
/* gas conserved variables (src/athena.hpp:52) */
enum { DUSTB_IDN = 0, DUSTB_IM1 = 1, DUSTB_IM2 = 2, DUSTB_IM3 = 3 };
/* <dust>/deposit */
enum { DUSTB_NGP = 0, DUSTB_CIC = 1, DUSTB_TSC = 2 };
/* <dust>/drag_solver (the point-particle solvers of SolveCoupledStage) */
enum { DUSTB_SOLVER_LOCAL = 0, DUSTB_SOLVER_APPLYA = 1, DUSTB_SOLVER_DC1 = 2,
       DUSTB_SOLVER_DC2 = 3 };
/* x3 physical boundary of the dust (x3bc_dust, src/bvals/bvals.hpp) */
enum { DUSTB_X3_PERIODIC = 0, DUSTB_X3_REFLECT = 1, DUSTB_X3_OUTFLOW = 2 };

/* device error word bits */
#define DUSTB_ERR_HALO      0x1u  /* particle outside its block's deposit halo (dust_pm.cpp:241) */
#define DUSTB_ERR_ROUTE     0x2u  /* particle more than one block away (bvals_part.cpp:245) */
#define DUSTB_ERR_NGHBR     0x4u  /* no neighbour block covers a crossing (bvals_part.cpp:394) */
#define DUSTB_ERR_PGID      0x8u  /* PGID outside the pack */
#define DUSTB_ERR_TSTOP     0x10u /* stopping time not finite and positive (dust_newdt.cpp:53) */
#define DUSTB_ERR_WINDOW    0x20u /* fused kernels: a particle outside its tile window */
#define DUSTB_ERR_TIMEOUT   0x40u /* a bounded wait on an asynchronous copy ran out.  The CTA
                                   * that gave up may leave a copy in flight into shared memory
                                   * that a later CTA on the same SM then uses: every output of
                                   * that launch and of the launches after it on the stream is
                                   * untrusted, and the host must discard the step (restore the
                                   * last good state) rather than continue from it */
#define DUSTB_ERR_POINT     0x80u /* point-particle fields: invalid mass, owner, position or
                                   * TSC support (dust_gravity_points.cpp:29-33) */
#define DUSTB_ERR_CLOUD     0x100u /* refinable clouds: a cloud code with lobe bits (transition
                                    * clouds of refined meshes) or a cloud outside its block */

/* host return codes */
#define DUSTB_OK          0
#define DUSTB_EINVAL     (-1)
#define DUSTB_ELAUNCH    (-2)
#define DUSTB_ESCRATCH   (-3)
#define DUSTB_EUNSUP     (-4)

typedef struct dustb_mesh {
  int nmb;                 /* MeshBlocks in the pack (nmb_thispack) */
  int gids;                /* gid of the pack's first MeshBlock */
  int nx1, nx2, nx3;       /* active cells per MeshBlock */
  int ng;                  /* ghost cells (>= 2, src/dust/dust.cpp:325-330) */
  int multi_d, three_d;
  int x3bc;                /* DUSTB_X3_* */
  double x1min, x1max, x2min, x2max, x3min, x3max;   /* mesh_size */
  const double *mb_size;   /* nmb x 9 */
  const int *nghbr;        /* nmb x 27 */
  /* shear-periodic x1 faces (3-D shearing box, <mesh>/ix1_bc = shear_periodic); 0: off.
   * nghbr keeps the plain periodic x1 neighbours; the shear maps the faces onto each other
   * shifted in x2 by the shear offset q Omega Lx time. */
  int shear_x1;
  int sb_nb2, sb_nb3;      /* MeshBlocks of one radial face along x2 and x3 */
  const int *sb_gid;       /* 2 x sb_nb3 x sb_nb2: gid of the face block (0 inner, 1 outer)
                              at (b3, b2) (the ShearingBox x1 boundary maps, bvals_part.cpp
                              sgid_map) */
  double time;             /* mesh time of the cycle (the offset of every stage's remaps) */
  /* refined meshes (blocks of several levels, 3-D); both NULL on a single-level mesh.  With
   * them dustb_route hands particles to neighbours of any level, the deposits are exchanged by
   * dustb_ghost_add_plan, the gathered fields by dustb_ghost_copy_ml, the mixed form takes the
   * plan and the coarse scratch in dustb_mixed_params, and the entry points that assume one
   * level (dustb_ghost_add, dustb_ghost_copy, dustb_dc1_sweep, the single-level cycles) return
   * DUSTB_EUNSUP. */
  const int *mb_lev;       /* nmb: level of each block (pmb->mb_lev) */
  const int *nghbr_ml;     /* nmb x 56: gid in every NeighborIndex slot of pmb->nghbr (four
                              sub-slots per face, two per edge, one per corner;
                              src/mesh/nghbr_index.hpp:20-60), -1 where the slot is empty */
  /* refinable clouds on a refined 3-D mesh: the leaf traversal's block geometry (a host struct
   * of device arrays, below); NULL: the clouds' uniform-mesh traversal */
  const struct dustb_leaf_tables *leaf;
} dustb_mesh;

/* The block geometry of the refinable clouds' leaf traversal on a refined 3-D mesh
 * (DustGasDrag::BuildLeafTraversal3D, src/dust/dust_cloud3d.cpp:357-860, one rank: block slot =
 * gid - gids), built on the host by dustb_host_leaf_tables (athenak_b200/host/leaf_tables.hpp).
 * Every pointer is a device array.  A uniform mesh is the case nlev = 0. */
#define DUSTB_LEAF_MAXNB 64
typedef struct dustb_leaf_tables {
  int nlev;                /* max_level - root_level */
  int nfine[3];            /* the domain in cells of the finest level */
  double root_dx[3];       /* the root level's cell size (mesh extent / mesh cells): a level-L
                              cloud's half-width is root_dx / 2^L */
  const int *fbox;         /* nmb x 6: [x0, x1) x [y0, y1) x [z0, z1) in finest cells */
  const int *blev;         /* nmb: level above the root */
  const int *nnb;          /* nmb: distinct neighbours */
  const int *nb;           /* nmb x 64: their block slots, in NeighborIndex slot order */
  const int *nbs;          /* nmb x 64 x 3: the shift (in domain lengths) of each: the
                              neighbour's image next to the block is the block moved by -shift */
  const int *nbmax;        /* nmb: the finest level among a block and its neighbours */
  const int *safe;         /* nmb x 3: the ring (finest cells) the neighbours certainly hold */
  const long long *lockey; /* nmb: logical-location keys (level << 57 | lx3 << 38 | lx2 << 19 |
                              lx1), ascending */
  const int *locblk;       /* nmb: the block of each key */
  /* the scratch of the clouds' multilevel u* copy exchange (dustb_ghost_copy_ml for 3
   * variables: dustb_ghost_copy_ml_bytes) used by the cloud calls that exchange u* */
  double *coarse;
  long long coarse_bytes;
} dustb_leaf_tables;

typedef struct dustb_particles {
  double *pr;              /* 17 x stride */
  int *pi;                 /* 5 x stride */
  long long stride;        /* allocated capacity (row stride) */
  int npart;               /* live particles (nprtcl_thispack) */
} dustb_particles;

typedef struct dustb_fields {
  double *u0, *u1;         /* gas conserved state and its stage register */
  int nvar_gas;            /* 4 (isothermal) or 5 */
  double *qdep;            /* 5 vars: Q, P1..P3, pc2 rate */
  double *ustar;           /* 3 vars */
  double *dmom;            /* 3 vars */
  double *resid;           /* 4 vars (imex_resid) */
  double *work;            /* 3 vars (solver_ap) */
} dustb_fields;

typedef struct dustb_physics {
  int scheme;              /* DUSTB_NGP / CIC / TSC */
  int back_reaction;
  int consistent_gas;      /* <dust>/imex_consistent_gas (default on) */
  int drag_solver;         /* DUSTB_SOLVER_* */
  int shearing_box;        /* rotation and shear terms in the push */
  int stratified;          /* vertical gravity -Omega^2 z */
  int pc2_feedback_damping;
  double qshear, omega0, const_accel_phi;
  int x3_deposit_drop;     /* physical x3 faces (mesh.x3bc != periodic): 0 folds the ghost-cell
                              deposits beyond a face back into the mirrored active cells
                              (<dust>/x3_ghost_deposit = fold, the default), 1 drops them
                              (= drop); src/dust/dust.cpp:1323-1333,
                              src/bvals/bvals_dep_general.cpp:130-140 */
} dustb_physics;

typedef struct dustb_ctx {
  dustb_mesh mesh;
  dustb_particles part;
  dustb_fields f;
  dustb_physics phys;
  unsigned int *err;       /* device error word */
} dustb_ctx;

/* ---- library ------------------------------------------------------------------------ */
int dustb_version(void);
/* Last CUDA error string of this library's host code (not thread safe). */
const char *dustb_last_error(void);

/* ---- FP64 per-task entry points (reference layout, straightforward kernels) ---------- */

/* DustGasDrag::FirstTwoImpRK stage 1 (src/dust/dust_push.cpp:63-79): u1 <- u0 (ghosts
 * included), particle registers (X1,V1) <- (X,V). */
int dustb_register_copy(const dustb_ctx *ctx, void *stream);

/* Harness stand-in for Hydro::RKUpdate with a zero flux divergence (the gas update is not
 * part of the drag step): u0 <- gam0 u0 + gam1 u1 over active cells, all gas variables. */
int dustb_gas_rk_noflux(const dustb_ctx *ctx, double gam0, double gam1, void *stream);

/* DustGasDrag::AddDragHistoryGas (src/dust/dust_pm.cpp:721-742): u0.m += atw_dt dmom. */
int dustb_history_gas(const dustb_ctx *ctx, double atw_dt, void *stream);

/* DustGasDrag::ExplicitPush, imex branch (src/dust/dust_push.cpp:249-297). */
int dustb_push_imex(const dustb_ctx *ctx, double gam0, double gam1, double beta_dt,
                    double atw_dt, void *stream);

/* ParticlesBoundaryValues::SetNewPrtclGID on a single-level mesh (src/bvals/bvals_part.cpp:
 * 115-429): x3 reflect/outflow, snap into [xmin, xmax), new PGID from the neighbour table,
 * periodic wrap of X and the RK registers.  x3_removed (2 doubles: mass, count) may be NULL
 * unless mesh.x3bc == DUSTB_X3_OUTFLOW. */
int dustb_route(const dustb_ctx *ctx, double *x3_removed, void *stream);

/* DustGasDrag::DepositDrag, imex scatter (src/dust/dust_pm.cpp:197-277): zero qdep, then
 * Q += m c W/V, P += m c W v/V with c = a_dt/(t_s + a_dt), y weights at y + sh x. */
int dustb_deposit_qp(const dustb_ctx *ctx, double a_dt, double sh, void *stream);

/* MeshBoundaryValuesDep::PackAndSendDeposit + RecvAndSumDeposit on one device
 * (src/bvals/bvals_dep.cpp:320-560): the ghost-cell deposits of every block are added into
 * the active strips of its neighbours, buffers in NeighborIndex order.  At physical x3 faces
 * the ghost deposits beyond the face are folded back into the mirrored active cells (ghost
 * plane ks-1-t into ks+t), those of the block's own column first, then those of its x1/x2
 * neighbours' ghost strips in NeighborIndex order (the reference's general remap,
 * DepRemapPlan with x3mode fold, bvals_dep_general.cpp:130-140), or dropped. */
int dustb_ghost_add(const dustb_ctx *ctx, double *field, int nvar, void *stream);

/* MeshBoundaryValuesCC::PackAndSendCC + RecvAndUnpackCC on one device (same-level copy
 * exchange), followed by DustGasDrag::UstarX3BCs at physical x3 faces when x3_bcs != 0
 * (src/dust/dust_tasks.cpp:445-469). */
int dustb_ghost_copy(const dustb_ctx *ctx, double *field, int nvar, int x3_bcs, void *stream);

/* The additive ghost-deposit exchange of a 3-D mesh with refinement levels: the static part
 * of the reference's general remap (DepRemapPlan, src/bvals/bvals_dep_general.cpp:1-35; the
 * apply is GeneralApply, :1135-1175).  Every ghost cell of every block is given to the active
 * cells it overlaps, weight = overlap volume / target cell volume measured in finest-level
 * cells, so the remap conserves the deposit exactly at any level difference; beyond a physical
 * x3 face a ghost cell is mirrored back (fold) or dropped.  The plan is built on the host (the
 * C++ host layer's dustb_host_dep_plan, athenak_b200/host/dep_plan.hpp) from the blocks'
 * logical locations and neighbour slots; its arrays are DEVICE arrays.  Cells are flat indices
 * m * (n3 n2 n1) + (k n2 + j) n1 + i of the padded block arrays. */
typedef struct dustb_dep_plan {
  int nseg;                /* target cells that receive deposits */
  const int *seg_tgt;      /* nseg target cells, ascending */
  const int *seg_ptr;      /* nseg + 1: the sources of target s are entries seg_ptr[s] .. */
  const int *ent_src;      /* source ghost cell of each entry, by (source gid, source cell) */
  const double *ent_w;     /* overlap volume / target cell volume */
} dustb_dep_plan;
/* field (nmb, nvar, n3, n2, n1): target += sum over its entries of w * source, summed in
 * entry order and added once (the reference's order; FP64, bit-reproducible). */
int dustb_ghost_add_plan(const dustb_ctx *ctx, const dustb_dep_plan *plan, double *field,
                         int nvar, void *stream);

/* The copy exchange of a cell-centred field on a refined 3-D mesh (ctx->mesh.nghbr_ml and
 * mb_lev set; periodic; even nx and ng, nx >= 2 ng): AthenaK's multilevel boundary values as
 * the dust module's u* exchange uses them (DustGasDrag::SendUstar / RecvUstar /
 * FinishUstarGhosts, src/dust/dust_tasks.cpp:262-442): restriction into every block's coarse
 * array (MeshRefinement::RestrictCC), the exchange with same-level, coarser and finer
 * neighbours in the index boxes of MeshBoundaryValuesCC::InitSendIndices / InitRecvIndices
 * (src/bvals/buffs_cc.cpp), FillCoarseInBndryCC and the min-mod ProlongateCC
 * (src/bvals/prolongation.cpp, src/mesh/prolongation.hpp).  coarse: device scratch of
 * dustb_ghost_copy_ml_bytes (the coarse arrays, cleared at every call). */
long long dustb_ghost_copy_ml_bytes(const dustb_mesh *mesh, int nvar);
int dustb_ghost_copy_ml(const dustb_ctx *ctx, double *field, int nvar, double *coarse,
                        long long coarse_bytes, void *stream);

/* GasImplicitSolve's per-cell solve (dust_pm.cpp:426-436 and the dc1 local guess,
 * dust_solver.cpp:643-649): ustar = (u0.m + P)/(rho + Q) over active cells. */
int dustb_solve_ustar(const dustb_ctx *ctx, void *stream);

/* One ApplyDefectCorrection sweep on ustar (dust_solver.cpp:226-252): ghost fill of ustar,
 * operator gather/deposit into work, additive ghost exchange of work, per-cell correction. */
int dustb_dc1_sweep(const dustb_ctx *ctx, double a_dt, double sh, void *stream);

/* DustGasDrag::GatherKickPMBR (dust_pm.cpp:450-568): zero dmom; gather u*, kick, record
 * R = dv/a_dt, deposit -m W dv / V into dmom with the same weights. */
int dustb_gather_kick_pmbr(const dustb_ctx *ctx, double a_dt, double sh, void *stream);

/* DustGasDrag::ApplyPMBR imex (dust_pm.cpp:605-711): the consistent point split when
 * phys.consistent_gas, else u0.m += dmom and dmom /= a_dt. */
int dustb_apply_pmbr(const dustb_ctx *ctx, double a_dt, void *stream);

/* DustGasDrag::NewTimeStep (src/dust/dust_newdt.cpp:108-149): *dt_out (device double) =
 * dt_cfl * min over particles of dx/|v| (the y transport velocity includes -q Omega x in
 * a 3-D shearing box).  Written on the device; no host wait. */
int dustb_newdt(const dustb_ctx *ctx, double dt_cfl, double *dt_out, void *stream);

/* Stopping-time validation and extrema of RefreshStoppingTimeMaximum
 * (dust_newdt.cpp:34-98): out[0] = max t_s (DBL_MAX if any is invalid), out[1] = min t_s. */
int dustb_tstop_extrema(const dustb_ctx *ctx, double *out, void *stream);

/* ---- cell index and sort (src/dust/dust_cloud_device.cpp:1881-1977) ------------------ */

/* Scratch bytes of dustb_cell_index / dustb_sort_by_cell for npart particles. */
long long dustb_sort_scratch_bytes(const dustb_mesh *mesh, int npart);

/* The particles' cell keys m*ncell + (k nx2 + j) nx1 + i with the floor() cell formula of
 * SortParticles, and their order: order[0..npart) lists the particles sorted by
 * (key, index), cstart[0..nmb*ncell] the first position of every cell (a CSR over cells). */
int dustb_cell_index(const dustb_ctx *ctx, int *order, int *cstart, void *scratch,
                     long long scratch_bytes, void *stream);

/* DustGasDrag::SortParticles: every particle row moved into the spare arrays (same
 * stride) in (block, k, j, i, old index) order.  The caller swaps the arrays, as the
 * reference does with sort_spare_r/i. */
int dustb_sort_by_cell(const dustb_ctx *ctx, double *spare_pr, int *spare_pi, void *scratch,
                       long long scratch_bytes, void *stream);

/* Fixed size of the device array behind dustb_cell_index_static. */
#define DUSTB_STATIC_SCRATCH_BYTES (32ll << 20)

/* dustb_cell_index for callers that cannot allocate device memory when they call it: a host
 * code whose device memory all comes from its own pool reserved at start-up, or one that
 * must not make the synchronising cudaMalloc / cudaFree calls inside its time step.  The
 * outputs are those of dustb_cell_index; the scratch is a file-scope device array of
 * DUSTB_STATIC_SCRATCH_BYTES (32 MiB), which every GPU that loads the library holds until the
 * process exits.  No counterpart in the reference (its sort allocates through Kokkos and
 * thrust).
 *  - Inputs that need more scratch than the array (4 bytes per particle plus 4 per cell plus
 *    a little) are rejected with DUSTB_ESCRATCH before anything runs; dustb_last_error()
 *    names the sizes.
 *  - The first call on a device looks up the array's device address (cudaGetSymbolAddress,
 *    with that device current); make that first call before any stream capture.
 *  - Every call shares the one array: calls that may overlap on the GPU (on different
 *    streams without ordering between them) race and must not be issued.  Nothing in the
 *    array needs to start at zero; each call writes what it reads.
 *  - It calls no cudaMalloc, cudaFree or allocating library routine.
 *  - The looked-up address does not survive cudaDeviceReset (which unloads the module): a
 *    caller that resets a device calls dustb_cell_index_static_reset() before its next call. */
int dustb_cell_index_static(const dustb_ctx *ctx, int *order, int *cstart, void *stream);
/* Forgets the device addresses dustb_cell_index_static looked up (after a cudaDeviceReset);
 * the next call on each device looks its address up again.  Not while calls are running. */
int dustb_cell_index_static_reset(void);

/* ---- the cloud order index (DustGasDrag::UpdateCloudOrder, src/dust/dust_cloud_device.cpp:
 * 1992-2055; the identity after a sort, :1956-1975) -------------------------------------
 * An index of the particles in (block, k, j, i, index) order without moving them, and the
 * 64-bit tag (PTAG the low word, PTAGH the high) of the particle each slot indexed, so that a
 * later check finds any reordering of the rows.  The keys are those of dustb_cell_index.
 * The host keeps the reference's control (rebuild every cloud_order_interval cycles, after a
 * failed check, or when the index is longer than the particle set; none after a sort in the
 * same cycle; no index below 2 particles). */
/* Rebuild: ord[0..npart), tag[0..npart); scratch as dustb_sort_scratch_bytes. */
int dustb_cloud_order(const dustb_ctx *ctx, int *ord, unsigned long long *tag, void *scratch,
                      long long scratch_bytes, void *stream);
/* After a sort in cell order: ord[k] = k and its tag (:1970-1972). */
int dustb_cloud_order_identity(const dustb_ctx *ctx, int *ord, unsigned long long *tag,
                               void *stream);
/* The check between rebuilds (:2001-2010): *bad (device int) = the entries k < n whose ord[k]
 * is outside [0, npart) or whose particle's tag is not tag[k]. */
int dustb_cloud_order_check(const dustb_ctx *ctx, const int *ord, const unsigned long long *tag,
                            int n, int *bad, void *stream);

/* ---- point-particle fields for self-gravity and outputs (src/dust/dust_gravity_points.cpp)
 * 3-D point particles on a uniform mesh (PointGravityTransferSupported, :162-167).  Fields
 * have the mesh layout (nmb, nvar, n3, n2, n1); halo is a scratch field of the same shape.
 * The ghost deposits are remapped as the drag's are (same-level neighbours, shear-periodic x1
 * faces), except that at physical x3 faces they are always folded (the transfers' own plans,
 * :176-178).  A rejected particle sets DUSTB_ERR_POINT and contributes nothing. */
/* DepositPointGravityDensity (:215-249): owned (nvar 1) = the TSC density m W / V on the
 * active cells, the ghost cells zero.  Needs scheme TSC (EUNSUP otherwise). */
int dustb_point_gravity_density(const dustb_ctx *ctx, double *owned, double *halo, void *stream);
/* GatherPointGravityAcceleration (:316-369): acc[d * acc_stride + p] (d = 0..2, acc_stride >=
 * npart) = the TSC weights of particle p over the force field, whose active cells are owned
 * (nvar 3) and whose ghost cells take, by the transpose of the deposit remap (GatherMap
 * :121-160), the owned values of the cells their deposits land in.  halo: nvar 3. */
int dustb_point_gravity_gather(const dustb_ctx *ctx, const double *owned, double *halo,
                               double *acc, long long acc_stride, void *stream);
/* DepositPointScienceFields (:257-305): out (nvar 4, or 1 with mass_only) = m W / V and
 * m v W / V with the coupling's weights (ctx scheme) on the active cells, the ghost cells zero;
 * species >= 0: that species only.  halo: the same nvar. */
int dustb_point_science_fields(const dustb_ctx *ctx, double *out, double *halo, int mass_only,
                               int species, void *stream);

/* ---- refinable clouds on a uniform 2-D or 3-D mesh (src/dust/dust_imex3d.cpp) ----------
 * Plain P1 hat clouds: PLEV holds the cloud level L (half-width dx / 2^L along each
 * direction), integrated exactly over the cells of the block and its same-level neighbours
 * (CloudShape1D, LeafTraversal3D::ForEach / LeafTraversal::ForEach on a uniform mesh; 2-D:
 * the LeafApi<LeafTraversal> forms).  At physical x3 faces the part of a cloud beyond the face
 * comes back mirrored about it; shear-periodic x1 faces: EUNSUP.  A cloud code with lobe bits
 * (the transition clouds of refined meshes) or a cloud outside its block sets DUSTB_ERR_CLOUD
 * and is skipped. */
/* CloudDepositImplicitT (:61-99): qdep cleared, then Q = m c W / V and P = Q v into the owner
 * cells (no ghost exchange needed). */
int dustb_cloud_deposit_qp(const dustb_ctx *ctx, double a_dt, double sh, void *stream);
/* Bytes of the gather pack (12 doubles per padded cell, PackGatherField3D). */
long long dustb_cloud_gpack_bytes(const dustb_mesh *mesh);
/* CloudGatherImplicit3D's plain kernel (CloudGatherKickT, :114-175): u* (ghost cells filled by
 * the caller's copy exchange) packed with its central differences into gpack, the linear-
 * moment gather, the kick (v, R), and with back-reaction the impulse into dmom (cleared). */
int dustb_cloud_gather_kick(const dustb_ctx *ctx, double a_dt, double sh, double *gpack,
                            void *stream);
/* CloudDefectCorrection (src/dust/dust_imex3d_dc.cpp:229-274), one sweep: the u* copy
 * exchange, its pack, the clouds' operator D M G x (CloudOperatorKernelT) into work, then
 * x += (rho + Q)^-1 (M + P - rho x - D M G x) on the active cells. */
int dustb_cloud_dc1_sweep(const dustb_ctx *ctx, double a_dt, double sh, double *gpack,
                          void *stream);
/* ApplyPMBR for the clouds: with consistent_gas the overlap split
 * (CloudImplicitConsistencyOverlapT, src/dust/dust_imex3d.cpp:669-790; the residual in
 * resid), otherwise the plain PMBR. */
int dustb_cloud_apply_pmbr(const dustb_ctx *ctx, double a_dt, double sh, void *stream);
/* The clouds' pc2 (src/dust/dust_cloud3d.cpp:1362-1538): CloudPredictorT (qdep cleared, the
 * step-start gas velocity m / rho of u1 put in work and packed, the linear gather, the drag
 * impulse -dt (m / t_s)(ubar - v) into qdep 1-3 and, with rate_dep, m / t_s into qdep 4 of the
 * owner cells) and CloudAdvanceT (u* packed, the midpoint gather from the registers X1, V1,
 * the implicit-midpoint kick and drift of CloudPC2Push, the impulse into dmom, cleared). */
int dustb_cloud_pc2_predictor(const dustb_ctx *ctx, double dt, int rate_dep, double *gpack,
                              void *stream);
int dustb_cloud_pc2_advance(const dustb_ctx *ctx, double dt, double *gpack, void *stream);
/* (dustb_cloud_imex_cycle, dustb_cloud_pc2_cycle: with the fused cycles below) */

/* ---- refinable clouds on a refined 3-D mesh (mesh.leaf set) ---------------------------
 * The calls above then integrate every cloud over the actual leaves (LeafTraversal3D::ForEach,
 * src/dust/dust_leaf3d.hpp:368-513): the half-width root_dx / 2^L of its level L, the transition
 * lobes of its code (bits 6-7 x1, 4-5 x2, 9-10 x3: CloudShape1D, src/dust/dust.hpp:240-298), the
 * cells of its block when the support lies inside it, else of the block and its distinct
 * neighbours when they cover the support (the safe ring or the band scan, NeedGlobal / Covered),
 * else of every block whose periodic image meets it; gathers with the point rule along lobed
 * directions (GatherCode).  Periodic x1 and x2; x3 periodic or physical (the mirrored part);
 * u* exchanges by dustb_ghost_copy_ml with leaf->coarse.
 *
 * The split's controls (<dust>/cloud_split_*, src/dust/dust_cloud.cpp:140-270). */
typedef struct dustb_cloud_split {
  int max_level;           /* clouds are never split beyond this level (cloud_max_level: nlev, or
                              cloud_split_max_level when that is lower) */
  int split_everywhere;    /* test_cloud_split_everywhere: split regardless of the mesh */
  int split_overlap;       /* 1 (default): split once the shrunk support meets finer leaves; 0:
                              once it lies entirely on them */
  int split_buffer;        /* test_cloud_split_buffer: the finer leaves of level l dilated by
                              buffer << (nlev - l + 1) finest cells (0: none) */
  double slack;            /* cloud_split_slack (0.02): the support shrunk by this fraction */
  long long budget;        /* cloud_split_budget (0: none): the split events are taken in
                              particle order while the pieces appended before them stay below
                              the budget (the first is always taken, so at most 26 pieces
                              beyond it); the later events wait for a later call */
} dustb_cloud_split;
/* CloudInstantSwitch (src/dust/dust_cloud.cpp:1023-1085): every plain cloud of level >= L takes
 * the level max(L, level of the leaf holding its centre); lobed clouds and clouds whose leaf is
 * not found keep theirs.  *nchange (host) receives the clouds changed (the call synchronizes
 * the stream).  scratch: 4 bytes. */
int dustb_cloud_instant_switch(const dustb_ctx *ctx, int level_cap, int *nchange, void *scratch,
                               void *stream);
/* Bytes of scratch for dustb_cloud_split_p1 with npart particles. */
long long dustb_cloud_split_scratch_bytes(int npart);
/* SplitCloudsP1DeviceT (src/dust/dust_cloud3d.cpp:1005-1310) without the split velocity and
 * the block marks: a plain cloud whose (shrunk) support meets (or lies on) finer
 * leaves, or a lobed cloud whose lobe side became eligible, is split along each direction into
 * the P1 pieces of its separation flags (centre child with the lobes kept, edge children at
 * +-half-width with a quarter of the parent's shape each); pieces other than the centre are
 * appended after the live particles with the parent's rows, tags tag0, tag0 + 1, ... in the
 * order of the exclusive scan; each piece's position (wrapped; mirrored with its x3 lobe at a
 * physical x3 face, vz flipped at a reflecting one), mass, code and block (its owner leaf's, or
 * the parent's when none is found).  *nnew (host) receives the pieces appended (the call
 * synchronizes); the caller adds them to npart.  DUSTB_ESCRATCH when npart + new pieces exceed
 * the particle capacity (nothing written; *nnew holds the count). */
int dustb_cloud_split_p1(const dustb_ctx *ctx, const dustb_cloud_split *split,
                         unsigned long long tag0, int *nnew, void *scratch, long long bytes,
                         void *stream);

/* ---- the particle science file (pbin, src/outputs/pbin.cpp): its device side -----------
 * The host writes the file (athenak_b200/host/pbin.hpp); these calls find the active rows
 * and pack their columns. */
typedef struct dustb_pbin_stats {
  long long active_rows;        /* mass != 0 (written) */
  long long zero_mass_rows;     /* mass == 0 (outflow tombstones, left out) */
  long long invalid_mass_rows;  /* active rows whose mass is not finite or not > 0 */
  long long negative_tag_rows;  /* active rows with PTAGH < 0 (tags >= 2^63) */
  long long differ_rows;        /* active rows whose species is not 0 or t_s not ts0 */
  double mass_min, mass_max;    /* over the active rows (fmin / fmax: NaN skipped) */
} dustb_pbin_stats;
/* the particle columns, in the file's order */
enum { DUSTB_PBIN_ID = 0, DUSTB_PBIN_SPECIES = 1, DUSTB_PBIN_X1 = 2, DUSTB_PBIN_X2 = 3,
       DUSTB_PBIN_X3 = 4, DUSTB_PBIN_V1 = 5, DUSTB_PBIN_V2 = 6, DUSTB_PBIN_V3 = 7,
       DUSTB_PBIN_MASS = 8, DUSTB_PBIN_STOPPING_TIME = 9 };
long long dustb_pbin_scratch_bytes(int npart);
/* ParticleBinaryOutput::LoadOutputData (:394-420) and the checks of WriteOutputFile
 * (:526-560): idx[0..active_rows) = the rows with mass != 0 in array order; *stats (device)
 * the counts and the mass range (ts0: the t_s of species 0 for the constant check). */
int dustb_pbin_rows(const dustb_ctx *ctx, int *idx, dustb_pbin_stats *stats, double ts0,
                    void *scratch, long long scratch_bytes, void *stream);
/* PackParticleColumns (:322-390): column DUSTB_PBIN_* of rows idx[0..n) into out (device):
 * ID uint64 (PTAG low word, PTAGH high), SPECIES uint32, the reals float64 or, with single,
 * float32. */
int dustb_pbin_pack(const dustb_ctx *ctx, const int *idx, int n, int column, int single,
                    void *out, void *stream);
/* ShuffleDeflate's byte shuffle (:243-262) of rows values of itemsize bytes, chunk by chunk
 * of chunk_rows rows: out[chunk + k * rows_c + i] = in[chunk + i * itemsize + k]. */
int dustb_pbin_shuffle(const void *in, long long rows, int itemsize, long long chunk_rows,
                       void *out, void *stream);

/* ---- pc2 (src/dust/dust_pm.cpp:109-194, :374-405, :585-602; dust_push.cpp:37-61,
 * :99-247) ---------------------------------------------------------------------------- */
int dustb_pc2_predictor(const dustb_ctx *ctx, double dt, int rate_dep, void *stream);
/* chi_max (device double, may be NULL): max over active cells of dt*qdep4/rho
 * (UpdateStiffness), computed before the damping. */
int dustb_pc2_apply_predictor(const dustb_ctx *ctx, double dt, double *chi_max, void *stream);
int dustb_pc2_midpoint(const dustb_ctx *ctx, void *stream);
int dustb_pc2_advance(const dustb_ctx *ctx, double dt, void *stream);
int dustb_pc2_commit(const dustb_ctx *ctx, double wpred, void *stream);

/* ---- fused FP64 cycles: the reference's task order for one cycle ----------------------- */

typedef struct dustb_imex_coeffs {
  double gamma;            /* imex2+ singly-diagonal coefficient (1+1/sqrt 2 or 1/2) */
  double dt;               /* cycle time step */
  double sh[2];            /* ImplicitShearShift of working stages 1, 2 */
} dustb_imex_coeffs;

/* One imex2+ cycle of refinable clouds on a uniform 3-D mesh (the task order of
 * dustb_imex_cycle with dustb_cloud_deposit_qp, dustb_cloud_dc1_sweep, dustb_cloud_gather_kick
 * and dustb_cloud_apply_pmbr); gpack as dustb_cloud_gpack_bytes. */
int dustb_cloud_imex_cycle(const dustb_ctx *ctx, const dustb_imex_coeffs *coeffs, double *gpack,
                           double *x3_removed, void *stream);
/* One imex2+ cycle of refinable clouds on a refined 3-D mesh (mesh.leaf set): the order of
 * dustb_cloud_imex_cycle with the clouds' leaf deposits, the gas state exchanged by
 * dustb_ghost_copy_ml (coarse: its scratch for ctx->f.nvar_gas) and u* with leaf->coarse. */
int dustb_cloud_refined_imex_cycle(const dustb_ctx *ctx, const dustb_imex_coeffs *coeffs,
                                   double *gpack, double *coarse, long long coarse_bytes,
                                   double *x3_removed, void *stream);
/* One pc2 cycle of the clouds (the order of dustb_pc2_cycle with the cloud predictor and
 * advance; chi_max as there). */
int dustb_cloud_pc2_cycle(const dustb_ctx *ctx, double dt, double *chi_max, double *gpack,
                          double *x3_removed, void *stream);

/* One imex2+ cycle of the drag step (stages 1 and 2; stage 3 is dormant): register copy,
 * gas stand-in, push, route, deposit, ghost add, solve (+dc1/dc2), ghost copy, gather-kick,
 * ghost add, apply, history.  x3_removed as in dustb_route. */
int dustb_imex_cycle(const dustb_ctx *ctx, const dustb_imex_coeffs *c, double *x3_removed,
                     void *stream);

/* ApplyDefectCorrection (src/dust/dust_solver.cpp:226-252), one dc1 sweep on a refined mesh:
 * u* exchanged by dustb_ghost_copy_ml (coarse: its scratch for 3 variables), the operator
 * D M G x of the point particles into work, its ghost deposits remapped by the plan
 * (dustb_ghost_add_plan), x += (rho + Q)^-1 (M + P - rho x - D M G x). */
int dustb_dc1_sweep_plan(const dustb_ctx *ctx, const dustb_dep_plan *plan, double a_dt,
                         double *coarse, long long coarse_bytes, void *stream);
/* One imex2+ cycle of the point-particle drag step on a refined 3-D mesh (ctx->mesh.nghbr_ml
 * and mb_lev set): the task order of dustb_imex_cycle with the deposits exchanged by
 * dustb_ghost_add_plan (plan: the mesh's general remap) and u*, the dc1 / dc2 operator's field
 * and the gas state by dustb_ghost_copy_ml (coarse: its scratch, sized for the gas state's
 * nvar_gas variables).  Periodic meshes, no implicit shear shift; the reference runs point
 * particles on refined 3-D meshes with amr_pic = instant_switch (src/dust/dust.cpp:1301-1340). */
int dustb_refined_imex_cycle(const dustb_ctx *ctx, const dustb_dep_plan *plan,
                             const dustb_imex_coeffs *c, double *coarse, long long coarse_bytes,
                             double *x3_removed, void *stream);

/* One pc2 cycle (integrator rk2): predictor, apply, gas tail, midpoint, advance, route,
 * ghost add, commit.  chi_max as in dustb_pc2_apply_predictor. */
int dustb_pc2_cycle(const dustb_ctx *ctx, double dt, double *chi_max, double *x3_removed,
                    void *stream);

/* DustGasDrag::ParticleHistory (src/dust/dust_science.cpp:391-482), the phst row, on a
 * single-level 3-D mesh of point particles.  row (device, 16 doubles): [0] particles with
 * m != 0, [1] mass, [2..4] momentum, [5] kinetic energy, [6] z_rms = sqrt(sum m z^2 / sum m),
 * each summed as the reference sums them (chunks of 4096 particles in particle order, then
 * the chunks in order: deterministic); [7] the largest density of the mass deposit on the
 * active cells (m/V with the deposit weights, the ghost deposits summed into their owners
 * as dustb_ghost_add sums them; among equal values the first cell in (block, k, j, i)
 * order), [8..10] that cell's centre, [11] its level above the root (0; with centre 0 and
 * -1 when the largest density is 0); [12] *chi_max when back_reaction (NULL or none: -1);
 * [13] -1 (no stiffness threshold); [14], [15] 0 (no coarsening events, no removal
 * counter).  The particle rows are read as they are (export the mixed shadow first).
 * Scratch: dustb_phst_scratch_bytes.  2-D meshes: DUSTB_EUNSUP. */
long long dustb_phst_scratch_bytes(const dustb_mesh *mesh, int npart);
int dustb_phst(const dustb_ctx *ctx, const double *chi_max, double *row, void *scratch,
               long long scratch_bytes, void *stream);

/* ---- mixed-precision form ---------------------------------------------------------------
 * A compact device shadow of the particles, kept between imports and exports: per particle
 * a packed cell id (block, k, j, i), FP32 offsets inside the cell, FP32 velocity, velocity
 * register, register displacement x1 - x (cells), drag rate, stopping time and mass.  The
 * gas and the deposit fields stay the reference's FP64 arrays of dustb_ctx (per-cell
 * accumulators, solves and the gas update in FP64); weights, gathers and kicks run in FP32
 * with the drag factor a/(t_s + a) formed in FP64.  The shadow is kept sorted by cell at
 * every stage (two copies; the push moves each particle to its slot in the other), so the
 * particles of a CTA's tile of cells are one contiguous range, copied into shared memory
 * with bulk copies.  One thread per source cell accumulates its particles' 27-point
 * deposits in registers; neighbouring threads combine the contributions that land on the
 * same cell and add them to the FP64 field.  All the workspace is the caller's
 * (dustb_mixed_workspace_bytes).
 * No reference counterpart: the reference keeps only the FP64 SoA. */

enum { DUSTB_MIXED_PROBE_COPY_TIMEOUT = 7 };
/* variant flag: the tile kernels as one CTA per tile instead of persistent CTAs taking the
 * tiles, heaviest first, from a device work queue (the default) */
#define DUSTB_MIXED_GRID_TILES 8
/* variant flag: the momentum ledgers off.  By default the kick tiles and the push return every
 * FP32 rounding of the gas-dust momentum exchange to the gas in FP64 (per tile, per CTA), so
 * that total gas + dust momentum is conserved to FP64 round-off; with this flag it is
 * conserved to the FP32 rounding of the exchange (about 1e-8 of the exchanged momentum per
 * cycle) and a cycle takes about 5 % less time */
#define DUSTB_MIXED_NO_LEDGER 16
/* variant flag (3-D): the gathering tiles (operator, kick, pc2 predictor and advance) stage
 * their gas window -- the tile's rows and one layer around them in three planes of the FP32
 * gather window -- in shared memory by one tensor copy (TMA) per tile, instead of every thread
 * loading its 27 cells from global memory.  Same results; off by default: on the 256^3
 * benchmark workload the per-thread loads (L1 hits, issued while the particle copies fly) are
 * faster (operator tile 5.7 against 7.1 ms, kick tile 8.3 against 10.0 ms per launch) */
#define DUSTB_MIXED_WINDOW_TMA 32

typedef struct dustb_mixed_params {
  double dx[3];            /* uniform cell size (single-level mesh) */
  int rows_per_tile;       /* 0: chosen by the library; else rows of nx1 cells per CTA tile */
  int chunk;               /* shared-memory columns per CTA pass (chunk - 8 particles per
                              pass), a multiple of 4 in 64..8192; 0: the largest that keeps
                              as many CTAs per SM as their registers allow (2380 for tiles
                              of 128 cells) */
  int variant;             /* 0, or any of DUSTB_MIXED_GRID_TILES, DUSTB_MIXED_NO_LEDGER,
                              DUSTB_MIXED_WINDOW_TMA;
                              DUSTB_MIXED_PROBE_COPY_TIMEOUT (with
                              or without the flag): a failure-detection test
                              hook (the first tile CTA 0 takes in every deposit launch never
                              issues its first copy: its bounded wait runs out, the CTA returns
                              and sets DUSTB_ERR_TIMEOUT) */
  double *x3_removed;      /* device (mass, count) of the particles removed at outflow x3
                              faces, accumulated; required when mesh.x3bc is
                              DUSTB_X3_OUTFLOW, else may be NULL */
  /* refined meshes (ctx->mesh.nghbr_ml set; periodic, imex2+ cycles): dx above is then the
   * root level's cell size, root_level the root level's number (the levels of mb_lev count
   * from it, at most 7 above it); plan the mesh's general deposit remap (dustb_ghost_add_plan)
   * and coarse / coarse_bytes the scratch of dustb_ghost_copy_ml for ctx->f.nvar_gas
   * variables.  All zero on a single-level mesh. */
  int root_level;
  const dustb_dep_plan *plan;
  double *coarse;
  long long coarse_bytes;
} dustb_mixed_params;

long long dustb_mixed_workspace_bytes(const dustb_mesh *mesh, int npart);

/* Detached rows: between an import and an export the mixed cycles (and the cell tasks they
 * call: dustb_solve_ustar, dustb_ghost_add, dustb_ghost_copy, dustb_gas_rk_noflux,
 * dustb_history_gas, dustb_pc2_apply_predictor, dustb_pc2_midpoint, dustb_pc2_commit) read no
 * particle row, so a host code may free the reference rows and pass ctx->part with
 * pr = pi = NULL and npart kept, holding only the shadow while the cycles run; import and
 * export need the rows attached (DUSTB_EINVAL otherwise). */

/* Builds the shadow of particles 0..npart-1 of ctx->part (positions, velocities, registers,
 * rates, t_s, m) and sorts it by cell. */
int dustb_mixed_import(const dustb_ctx *ctx, const dustb_mixed_params *mp, void *ws,
                       long long ws_bytes, void *stream);

/* Writes X, V, X1, V1, R and PGID of every shadow particle back into its reference row.
 * The last cycle's stage-2 consistent dust kick, which the shadow keeps pending until the
 * next cycle's push, is applied to the V and R written (ctx->f.resid as that cycle left it). */
int dustb_mixed_export(const dustb_ctx *ctx, const dustb_mixed_params *mp, void *ws,
                       long long ws_bytes, void *stream);

/* One imex2+ cycle of the drag step on the shadow (the same task sequence as
 * dustb_imex_cycle; the FP64 mesh fields of ctx are used and updated).  On a periodic mesh
 * the tiles gather from and deposit into the owning blocks' active cells directly; with
 * physical x3 faces or shear-periodic x1 faces they use each block's own ghost cells and the
 * FP64 ghost exchanges (dustb_ghost_add / dustb_ghost_copy: x3 fold or drop, shear remaps)
 * run around them.  The push routes particles as dustb_route does (x3 reflect / outflow,
 * shear-periodic crossings).  With an implicit shear shift (c->sh, 3-D shearing box) the
 * tiles place the weights at y + sh x; particles whose shifted position lies in the next
 * cell are sorted into an edge bin that per-particle kernels deposit and gather (2-D meshes
 * with sh != 0: DUSTB_EUNSUP, the FP64 form). */
int dustb_mixed_imex_cycle(const dustb_ctx *ctx, const dustb_mixed_params *mp, void *ws,
                           long long ws_bytes, const dustb_imex_coeffs *c, void *stream);

/* One pc2 cycle (integrator rk2) on the shadow, the task sequence of dustb_pc2_cycle: the
 * predictor tiles gather m/rho of u1 and deposit the predicted impulse and rate into qdep;
 * the FP64 cell passes apply it and form the midpoint u*; the particles are re-sorted by the
 * cell of their half-step gather position, where the advance tiles gather u*, solve the
 * implicit midpoint step (Coriolis, vertical gravity) and deposit the drag impulse into
 * dmom; particles whose gather position lies beyond a physical x3 face or a shear-periodic
 * x1 face are advanced by a per-particle kernel on their block's own ghost cells; then
 * every particle moves to its new position (routing as dustb_route) and is re-sorted.
 * chi_max as in dustb_pc2_apply_predictor (may be NULL).  The export writes X1 = X (the
 * half-step position register is not kept; the next cycle's register copy sets it).
 * On entry u0's ghost cells hold the copy exchange of the active cells (the state every
 * cycle leaves): on a periodic mesh the tiles read the gas through the owning blocks.
 * After imex cycles, export and import the shadow before the first pc2 cycle (the export
 * applies the imex cycle's pending consistent kick). */
int dustb_mixed_pc2_cycle(const dustb_ctx *ctx, const dustb_mixed_params *mp, void *ws,
                          long long ws_bytes, double dt, double *chi_max, void *stream);

/* The autotuner of the tile kernels: times the candidate tile shapes -- rows per tile (1,
 * 2, 4, 8 where they divide nx2 and give at most 256 cells), particles per pass (the default,
 * 2304, 4096, 4608) and the launch form (persistent CTAs on the device work queue or one CTA
 * per tile) -- with the Q/P and dc1 operator tiles on the caller's shadow and workspace as
 * they stand (after an import or a cycle), and writes the fastest into mp (rows_per_tile,
 * chunk, the DUSTB_MIXED_GRID_TILES flag of variant; *best_ms, if given, its time per Q/P +
 * operator pair).  It changes no particle or gas state: the tiles write only the stage
 * scratch fields qdep, the centre mass of imex_resid and work, which every cycle rewrites
 * before reading them.  Synchronous (it waits for its events); not inside a stream capture
 * and not while dustb_mixed_timing is on (DUSTB_EUNSUP).  The reference has no counterpart
 * (its kernels take Kokkos' default launch shapes); the counting sort has one bucket per
 * cell, so there is no sort-bucket width to tune. */
int dustb_mixed_tune(const dustb_ctx *ctx, dustb_mixed_params *mp, void *ws, long long ws_bytes,
                     double a_dt, double *best_ms, void *stream);

/* Re-sorts the shadow by cell (the SortParticles of the shadow; the reference rows keep
 * their order, export writes each particle back to its own row). */
int dustb_mixed_sort(const dustb_ctx *ctx, const dustb_mixed_params *mp, void *ws,
                     long long ws_bytes, void *stream);

/* Kernel timing of the mixed cycle: when enabled, the library records CUDA events around
 * every fused kernel it launches; dustb_mixed_kernel_times sums their durations (ms) and
 * launch counts per kernel id since the last reset (it synchronises the events).  The push
 * is two kernels: DUSTB_K_COUNT (the new cells and their histogram) and DUSTB_K_MOVE (the
 * push written to each particle's slot); DUSTB_K_CELLS holds the FP64 per-cell kernels and
 * exchanges, DUSTB_K_FILL the scan of the histogram, DUSTB_K_WINDOW the FP32 gather window
 * of a 3-D mesh written before each gathering tile launch. */
enum { DUSTB_K_COUNT = 0, DUSTB_K_FILL = 1, DUSTB_K_DEPOSIT_QP = 2, DUSTB_K_OPERATOR = 3,
       DUSTB_K_KICK = 4, DUSTB_K_CONSISTENT = 5, DUSTB_K_CELLS = 6, DUSTB_K_MOVE = 7,
       DUSTB_K_WINDOW = 8, DUSTB_K_NKERNELS = 9 };
int dustb_mixed_timing(int enable);
int dustb_mixed_kernel_times(double *ms, int *launches, int n);

/* ---- seeded synthetic inputs ----------------------------------------------------------- */

/* Parameters of the seeded uniform-random set-up (the hash placement of
 * src/pgen/dust_amr/dust_setup.hpp:36-50, :114-118; NSH drift dust_setup.hpp:58-65). */
typedef struct dustb_seed_desc {
  unsigned long long seed;
  int nspecies;                 /* <= 8 */
  int ppc[8];                   /* particles per cell of each species */
  double taus[8], mass[8];      /* stopping time and particle mass of each species */
  double vx[8], vy[8], vz[8];   /* mean velocity of each species */
  double vel_noise;             /* Gaussian sigma (Box-Muller on two hash draws) */
  double rho0, ug[3], gas_noise;/* gas density, velocity, uniform noise amplitude */
  int nb1, nb2, nb3;            /* MeshBlocks per direction (gid = (b3*nb2 + b2)*nb1 + b1) */
  /* the continuous size distribution (src/pgen/dust_amr/dust_setup.cpp:736-745): with
   * ts_lo > 0 species s is bin s of nspecies equal bins in ln t_s over [ts_lo, ts_hi], each
   * particle draws its t_s log-uniform inside its bin (taus[] unused) and weighs
   * mass[s] (t_s / t_mid)^mass_slope, t_mid the bin's geometric centre */
  double ts_lo, ts_hi, mass_slope;
  double hp;                    /* > 0: Gaussian heights of scale hp about x3 = 0 (redrawn
                                   while outside the mesh) in place of uniform x3 */
  int nsh;                      /* 1: every particle drifts at the NSH velocity of its own t_s
                                   (dust_setup.hpp:58-65) about the gas drift (ug[0], ug[1]);
                                   vx[], vy[] unused */
  double omega0, qshear;        /* (nsh) */
} dustb_seed_desc;

/* Fills particles 0..npart-1 (species blocks in order, tag = index) and the gas u0 (ghosts
 * included).  A test and benchmark input generator; the reference's problem generators are
 * the host code's own. */
int dustb_seed_uniform(const dustb_ctx *ctx, const dustb_seed_desc *desc, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DUSTB_H_ */
