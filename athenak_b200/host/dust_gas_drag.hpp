// dust_gas_drag.hpp -- the host side of the drag step in the reference's own terms.
//
// A DustGasDrag whose task functions carry the names, arguments and stage logic of the
// reference's (src/dust/dust_pm.cpp, dust_push.cpp, dust_solver.cpp, dust_newdt.cpp,
// src/bvals/bvals_part.cpp, src/dust/dust_cloud_device.cpp) and forward one for one to the
// C ABI of include/dustb.h on the pack's stream, plus the task list of one stage in the order
// AssembleDustGasDragTasks builds it (src/dust/dust_tasks.cpp:38-120), for one rank: the
// MPI send/receive pairs of the reference become the single-rank exchanges of the ABI, and
// the hydro's flux update is the ABI's zero-flux stand-in.  A failing call returns
// TaskStatus::fail with the library's message in LastError() (the reference aborts).
#ifndef ATHENAK_B200_DUST_GAS_DRAG_HPP_
#define ATHENAK_B200_DUST_GAS_DRAG_HPP_

#include <string>

#include "../../include/dustb.h"

namespace athenak_b200 {

// src/tasklist/task_list.hpp:32
enum class TaskStatus { fail, complete, incomplete };

// <dust>/coupling
enum class DustCoupling { imex, pc2 };

// The integrator state the drag tasks read: Driver::SetImEx2PlusCoefficients
// (src/driver/driver.cpp:278-300) and the mesh's time and step.
struct Driver {
  double gamma = 0.0;
  double gam0[3] = {0.0, 0.0, 0.0}, gam1[3] = {0.0, 0.0, 0.0}, beta[3] = {0.0, 0.0, 0.0};
  double a_twid[4][4] = {};
  double a_impl = 0.0;
  int nexp_stages = 2;           // stage 3 of imex2+ is dormant for the drag (dust.cpp:1646)
  double dt = 0.0, time = 0.0;   // Mesh::dt, Mesh::time
  int ncycle = 0;                // Mesh::ncycle
  void SetImEx2PlusCoefficients(double gamma_new);
};

class DustGasDrag {
 public:
  // ctx: the pack's arrays (device pointers, the reference's layout); stream: the pack's
  // (Kokkos default execution space) CUDA stream.  Allocates the few device scalars the
  // tasks write (the x3 outflow tally, the pc2 stiffness record, the new time step).
  DustGasDrag(const dustb_ctx &ctx, void *stream, DustCoupling coupling = DustCoupling::imex);
  ~DustGasDrag();
  DustGasDrag(const DustGasDrag &) = delete;
  DustGasDrag &operator=(const DustGasDrag &) = delete;

  dustb_ctx &Context() { return ctx_; }

  // ---- tasks of a stage (dust_tasks.cpp:56-107)
  TaskStatus FirstTwoImpRK(Driver *pdrive, int stage);     // dust_push.cpp:35-80
  TaskStatus RKUpdate(Driver *pdrive, int stage);          // Hydro::RKUpdate, zero flux
  TaskStatus AddDragHistoryGas(Driver *pdrive, int stage); // dust_pm.cpp:721-742
  TaskStatus ExplicitPush(Driver *pdrive, int stage);      // dust_push.cpp:99-297
  TaskStatus UpdateParticleGIDs(Driver *pdrive, int stage);// bvals_part.cpp:115-471
  TaskStatus DepositDrag(Driver *pdrive, int stage);       // dust_pm.cpp:104-277
  TaskStatus RecvDepQP(Driver *pdrive, int stage);         // bvals_dep.cpp:457-560
  TaskStatus GasImplicitSolve(Driver *pdrive, int stage);  // dust_pm.cpp:372-442
  TaskStatus RecvUstar(Driver *pdrive, int stage);         // the u* ghost copy (+ shear, x3)
  TaskStatus GatherKickPMBR(Driver *pdrive, int stage);    // dust_pm.cpp:450-568
  TaskStatus RecvPMBR(Driver *pdrive, int stage);          // the dmom deposit exchange
  TaskStatus ApplyPMBR(Driver *pdrive, int stage);         // dust_pm.cpp:576-711
  TaskStatus RecvU(Driver *pdrive, int stage);             // the hydro tail's u0 exchange
  TaskStatus NewTimeStep(Driver *pdrive, int stage);       // dust_newdt.cpp:108-149

  // SortParticles (dust_cloud_device.cpp:1881-1977): into the spare arrays, then swapped
  // in; the spares (same shape as the rows) become the caller's to keep or free.  With the
  // cloud order index on, the index becomes the identity, marked with the cycle ncycle.
  TaskStatus SortParticles(double *spare_pr, int *spare_pi, void *scratch, long long bytes,
                           int ncycle = -1);

  // UpdateCloudOrder (dust_cloud_device.cpp:1992-2055), <dust>/cloud_order_interval = n > 0:
  // an index of the particles in (block, cell, index) order without moving them, rebuilt
  // every n cycles, after a check finds a slot that no longer holds its particle, or when it
  // is longer than the particle set; kept as it is after a sort of the same cycle; none
  // below 2 particles.  Synchronises the stream for the check's count.  scratch: at least
  // dustb_sort_scratch_bytes.
  void SetCloudOrderInterval(int n) { cloud_order_interval_ = n; }
  TaskStatus UpdateCloudOrder(const Driver &drv, void *scratch, long long bytes);
  const int *CloudOrder() const { return cloud_ord_; }
  const unsigned long long *CloudOrderTags() const { return cloud_ord_tag_; }
  int CloudOrderLength() const { return cloud_ord_n_; }
  int CloudOrderBuilds() const { return cloud_ord_builds_; }

  // Point-particle fields (src/dust/dust_gravity_points.cpp) at the field time `time` (the
  // shear offset of the remap): the TSC density for self-gravity, the acceleration gathered
  // from an owned force field (acc row d at acc + d * acc_stride), and the mass and momentum
  // densities of the outputs.  halo: the caller's scratch field of the output's shape.
  TaskStatus DepositPointGravityDensity(double time, double *owned, double *halo);
  TaskStatus GatherPointGravityAcceleration(double time, const double *owned, double *halo,
                                            double *acc, long long acc_stride);
  TaskStatus DepositPointScienceFields(double time, double *out, double *halo, bool mass_only,
                                       int species);

  // <dust>/smr_transfer = refinable_cloud on a uniform 2-D or 3-D mesh (UsesRefinableClouds):
  // the deposit, the dc1 / dc2 sweeps, the gather-kick and the PMBR split of the imex tasks,
  // and the predictor and advance of pc2, run the clouds' kernels (PLEV = cloud level); their
  // deposits land in the owner cells, so the deposit exchanges are skipped.  Allocates the
  // gather pack.
  TaskStatus SetRefinableClouds(bool on);

  // A refined 3-D mesh (ctx.mesh.nghbr_ml and mb_lev set): the deposit exchanges by the general
  // remap of plan (MeshBoundaryValuesDep's general path; the plan's arrays stay the caller's),
  // the u* and gas-state copy exchanges by the multilevel exchange (RestrictCC, the 56-slot
  // boxes, ProlongCC) with scratch allocated here, the dc1 / dc2 sweeps with both.
  TaskStatus SetRefinedMesh(const dustb_dep_plan &plan);
  // Refinable clouds on a refined 3-D mesh: the leaf traversal's block geometry (a copy of the
  // struct, its device arrays the caller's; the u* exchange scratch allocated here), then
  // SetRefinableClouds(true).
  TaskStatus SetLeafTables(const dustb_leaf_tables &tables);
  // <dust>/cloud_split_*: the split's controls, cloud_split_enable (the P1 split of
  // RefineClouds), cloud_split_max_level = L (>= 0: the instant switch above L; the split
  // stops at L), and the next 64-bit tag of this rank (IssueTags' counter).
  void SetCloudSplit(const dustb_cloud_split &split, bool enable, int split_max_level,
                     unsigned long long next_tag);
  // RefineClouds (src/dust/dust_cloud.cpp:615-720), the task at the start of a cycle:
  // SplitAndMergeClouds (:984-988) -- the P1 split (pieces appended, npart and the tag counter
  // advanced), then the instant switch above cloud_split_max_level.  scratch: at least
  // dustb_cloud_split_scratch_bytes(npart).  The particle rows are the caller's: when the
  // pieces do not fit their capacity the task fails with the pieces' count in
  // LastSplitPieces(); the caller grows the rows (Context().part) and runs it again.
  TaskStatus RefineClouds(Driver *pdrive, void *scratch, long long bytes);
  unsigned long long NextTag() const { return next_tag_; }
  int LastSplitPieces() const { return last_split_; }
  int LastSwitched() const { return last_switch_; }

  // the stage's drag tasks in dependency order on one rank and one stream
  TaskStatus DoStage(Driver *pdrive, int stage);
  // one cycle: every working stage
  TaskStatus DoCycle(Driver *pdrive);

  // synchronises the stream and reads the device error word (nonzero: a particle the
  // reference would have aborted on)
  unsigned ErrorWord();
  // synchronises and reads the last NewTimeStep result, the pc2 stiffness record chi_max and
  // the x3 outflow tally (mass, count)
  double NewDt();
  double ChiMax();
  void X3Removed(double out[2]);
  const std::string &LastError() const { return last_error_; }

 private:
  TaskStatus Check(int rc, const char *task);
  dustb_ctx ctx_;
  void *stream_;
  DustCoupling coupling_;
  double *dev_scalars_ = nullptr;   // [0..1] x3 removed, [2] chi_max, [3] dt
  std::string last_error_;
  // the cloud order index (cloud_ord, cloud_ord_tag of the reference) and its control
  TaskStatus GrowCloudOrder();
  int *cloud_ord_ = nullptr;
  unsigned long long *cloud_ord_tag_ = nullptr;
  int *dev_bad_ = nullptr;
  int cloud_ord_cap_ = 0, cloud_ord_n_ = 0, cloud_sort_cycle_ = -1, cloud_ord_builds_ = 0;
  int cloud_order_interval_ = 0;
  bool clouds_ = false;
  double *gpack_ = nullptr;   // the clouds' gather pack (12 doubles per padded cell)
  // a refined mesh: the deposit remap and the copy exchange's scratch
  bool refined_ = false;
  dustb_dep_plan plan_{};
  double *coarse_ = nullptr;
  long long coarse_bytes_ = 0;
  // refinable clouds on a refined mesh: the leaf tables and the split's controls
  dustb_leaf_tables leaf_{};
  dustb_cloud_split split_{};
  bool split_enable_ = false;
  int split_max_level_ = -1, last_split_ = 0, last_switch_ = 0;
  unsigned long long next_tag_ = 0;
  int *dev_count_ = nullptr;
  TaskStatus CopyExchange(double *field, int nvar, int x3_bcs, const char *task);
};

// The mixed-precision form from the host (dustb_mixed_*): a compact FP32 shadow of the
// particles kept sorted by cell in a workspace this object allocates; Import after any change
// of the particle set, cycles, Export before anything reads the particle rows (outputs,
// restart, the FP64 task functions).  The mesh fields stay the pack's FP64 arrays.
class MixedDustGasDrag {
 public:
  // dx: the uniform cell size; rows_per_tile, chunk: the tile shape (0: the library's)
  MixedDustGasDrag(const dustb_ctx &ctx, void *stream, const double dx[3],
                   int rows_per_tile = 0, int chunk = 0);
  ~MixedDustGasDrag();
  MixedDustGasDrag(const MixedDustGasDrag &) = delete;
  MixedDustGasDrag &operator=(const MixedDustGasDrag &) = delete;

  TaskStatus Import();
  TaskStatus Export();
  // the library's autotuner on this workspace (after Import; synchronous, outside any stream
  // capture); ImexCycle and Pc2Cycle call it once themselves unless the tile shape was given
  TaskStatus Tune(double a_dt);
  TaskStatus ImexCycle(const Driver &drv);   // imex2+ (no implicit shear shift)
  TaskStatus Pc2Cycle(const Driver &drv);    // pc2
  dustb_ctx &Context() { return ctx_; }
  const std::string &LastError() const { return last_error_; }
  double ChiMax();                           // synchronises

 private:
  TaskStatus Check(int rc, const char *what);
  dustb_ctx ctx_;
  void *stream_;
  dustb_mixed_params mp_;
  bool tuned_ = false;
  void *ws_ = nullptr;
  long long ws_bytes_ = 0;
  double *dev_scalars_ = nullptr;            // [0..1] x3 removed, [2] chi_max
  std::string last_error_;
};

}  // namespace athenak_b200

#endif  // ATHENAK_B200_DUST_GAS_DRAG_HPP_
