// dust_gas_drag.cpp -- DustGasDrag's task functions forwarding to the C ABI (see the header).
#include "dust_gas_drag.hpp"

#include <cuda_runtime.h>

#include <cstring>

namespace athenak_b200 {

void Driver::SetImEx2PlusCoefficients(double gamma_new) {
  gamma = gamma_new;
  gam0[0] = 1.0; gam1[0] = 0.0; beta[0] = gamma;
  gam0[1] = (2.0 * gamma - 1.0) / (2.0 * gamma * gamma);
  gam1[1] = 1.0 - (2.0 * gamma - 1.0) / (2.0 * gamma * gamma);
  beta[1] = 1.0 / (2.0 * gamma);
  gam0[2] = 1.0; gam1[2] = 0.0; beta[2] = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int s = 0; s < 4; ++s) a_twid[i][s] = 0.0;
  a_twid[2][2] = (1.0 - 2.0 * gamma * gamma) / 2.0 / gamma;
  a_impl = gamma;
}

DustGasDrag::DustGasDrag(const dustb_ctx &ctx, void *stream, DustCoupling coupling)
    : ctx_(ctx), stream_(stream), coupling_(coupling) {
  if (cudaMalloc(&dev_scalars_, 4 * sizeof(double)) != cudaSuccess) {
    dev_scalars_ = nullptr;
    last_error_ = "DustGasDrag: device scalars not allocated";
    return;
  }
  cudaMemsetAsync(dev_scalars_, 0, 4 * sizeof(double), (cudaStream_t)stream_);
}

DustGasDrag::~DustGasDrag() {
  if (dev_scalars_) cudaFree(dev_scalars_);
  if (cloud_ord_) cudaFree(cloud_ord_);
  if (cloud_ord_tag_) cudaFree(cloud_ord_tag_);
  if (dev_bad_) cudaFree(dev_bad_);
  if (gpack_) cudaFree(gpack_);
  if (coarse_) cudaFree(coarse_);
  if (leaf_.coarse) cudaFree(leaf_.coarse);
  if (dev_count_) cudaFree(dev_count_);
}

// the copy exchange of a field: the multilevel one on a refined mesh
TaskStatus DustGasDrag::CopyExchange(double *field, int nvar, int x3_bcs, const char *task) {
  if (refined_) return Check(dustb_ghost_copy_ml(&ctx_, field, nvar, coarse_, coarse_bytes_, stream_), task);
  return Check(dustb_ghost_copy(&ctx_, field, nvar, x3_bcs, stream_), task);
}

TaskStatus DustGasDrag::SetRefinedMesh(const dustb_dep_plan &plan) {
  if (!ctx_.mesh.nghbr_ml || !ctx_.mesh.mb_lev) {
    last_error_ = "SetRefinedMesh: the mesh has no refinement tables (nghbr_ml, mb_lev)";
    return TaskStatus::fail;
  }
  const int nv = ctx_.f.nvar_gas > 5 ? ctx_.f.nvar_gas : 5;
  const long long bytes = dustb_ghost_copy_ml_bytes(&ctx_.mesh, nv);
  if (bytes <= 0) return Check(DUSTB_EINVAL, "SetRefinedMesh");
  if (!coarse_ || coarse_bytes_ < bytes) {
    if (coarse_) cudaFree(coarse_);
    if (cudaMalloc(&coarse_, (size_t)bytes) != cudaSuccess) {
      coarse_ = nullptr;
      last_error_ = "SetRefinedMesh: exchange scratch not allocated";
      return TaskStatus::fail;
    }
    coarse_bytes_ = bytes;
  }
  plan_ = plan;
  refined_ = true;
  return TaskStatus::complete;
}

TaskStatus DustGasDrag::SetLeafTables(const dustb_leaf_tables &tables) {
  leaf_ = tables;
  leaf_.coarse = nullptr;
  leaf_.coarse_bytes = 0;
  if (ctx_.mesh.nghbr_ml) {
    const long long bytes = dustb_ghost_copy_ml_bytes(&ctx_.mesh, 3);
    if (bytes <= 0 || cudaMalloc(&leaf_.coarse, (size_t)bytes) != cudaSuccess) {
      leaf_.coarse = nullptr;
      last_error_ = "SetLeafTables: exchange scratch not allocated";
      return TaskStatus::fail;
    }
    leaf_.coarse_bytes = bytes;
  }
  ctx_.mesh.leaf = &leaf_;
  return SetRefinableClouds(true);
}

void DustGasDrag::SetCloudSplit(const dustb_cloud_split &split, bool enable, int split_max_level,
                                unsigned long long next_tag) {
  split_ = split;
  split_enable_ = enable;
  split_max_level_ = split_max_level;
  next_tag_ = next_tag;
}

TaskStatus DustGasDrag::RefineClouds(Driver *pdrive, void *scratch, long long bytes) {
  if (!clouds_ || !ctx_.mesh.leaf) return TaskStatus::complete;
  last_split_ = last_switch_ = 0;
  if (split_enable_) {
    int nnew = 0;
    const int rc = dustb_cloud_split_p1(&ctx_, &split_, next_tag_, &nnew, scratch, bytes, stream_);
    last_split_ = nnew;
    if (rc != DUSTB_OK) return Check(rc, "RefineClouds");
    ctx_.part.npart += nnew;
    next_tag_ += (unsigned long long)nnew;
  }
  if (split_max_level_ >= 0) {
    if (!dev_count_ && cudaMalloc(&dev_count_, sizeof(int)) != cudaSuccess) {
      dev_count_ = nullptr;
      last_error_ = "RefineClouds: device counter not allocated";
      return TaskStatus::fail;
    }
    return Check(dustb_cloud_instant_switch(&ctx_, split_max_level_, &last_switch_, dev_count_,
                                            stream_),
                 "RefineClouds");
  }
  return TaskStatus::complete;
}

TaskStatus DustGasDrag::Check(int rc, const char *task) {
  if (rc == DUSTB_OK) return TaskStatus::complete;
  last_error_ = std::string(task) + ": " + dustb_last_error() + " (" + std::to_string(rc) + ")";
  return TaskStatus::fail;
}

// the implicit stage's a dt (a_impl dt) and the stage's RK weights, as the reference forms them
static inline double a_dt(const Driver *d) { return d->a_impl * d->dt; }

TaskStatus DustGasDrag::FirstTwoImpRK(Driver *pdrive, int stage) {
  // stage 1: the register copies; pc2 stage 2: the midpoint u* from the two gas states,
  // ghost cells included (dust_push.cpp:53-59)
  if (stage == 1) return Check(dustb_register_copy(&ctx_, stream_), "FirstTwoImpRK");
  if (coupling_ == DustCoupling::pc2 && stage == 2)
    return Check(dustb_pc2_midpoint(&ctx_, stream_), "FirstTwoImpRK");
  return TaskStatus::complete;
}

TaskStatus DustGasDrag::RKUpdate(Driver *pdrive, int stage) {
  const int s = stage - 1;
  if (coupling_ == DustCoupling::pc2)
    return Check(dustb_gas_rk_noflux(&ctx_, stage == 1 ? 1.0 : 0.5, stage == 1 ? 0.0 : 0.5, stream_),
                 "RKUpdate");
  return Check(dustb_gas_rk_noflux(&ctx_, pdrive->gam0[s], pdrive->gam1[s], stream_), "RKUpdate");
}

TaskStatus DustGasDrag::AddDragHistoryGas(Driver *pdrive, int stage) {
  if (coupling_ != DustCoupling::imex || stage != 2 || !ctx_.phys.back_reaction)
    return TaskStatus::complete;
  return Check(dustb_history_gas(&ctx_, pdrive->a_twid[stage][stage] * pdrive->dt, stream_),
               "AddDragHistoryGas");
}

TaskStatus DustGasDrag::ExplicitPush(Driver *pdrive, int stage) {
  const int s = stage - 1;
  if (coupling_ == DustCoupling::pc2) {
    if (stage != 2) return TaskStatus::complete;   // the advance of the midpoint stage
    if (clouds_)   // CloudAdvanceT (dust_cloud3d.cpp:1442-1536)
      return Check(dustb_cloud_pc2_advance(&ctx_, pdrive->dt, gpack_, stream_), "ExplicitPush");
    return Check(dustb_pc2_advance(&ctx_, pdrive->dt, stream_), "ExplicitPush");
  }
  const double atw = (stage == 2) ? pdrive->a_twid[stage][stage] * pdrive->dt : 0.0;
  return Check(dustb_push_imex(&ctx_, pdrive->gam0[s], pdrive->gam1[s], pdrive->beta[s] * pdrive->dt,
                               atw, stream_),
               "ExplicitPush");
}

TaskStatus DustGasDrag::UpdateParticleGIDs(Driver *pdrive, int stage) {
  if (coupling_ == DustCoupling::pc2 && stage != 2) return TaskStatus::complete;
  return Check(dustb_route(&ctx_, dev_scalars_, stream_), "UpdateParticleGIDs");
}

TaskStatus DustGasDrag::DepositDrag(Driver *pdrive, int stage) {
  if (!ctx_.phys.back_reaction) return TaskStatus::complete;
  if (coupling_ == DustCoupling::pc2) {
    if (stage != 1) return TaskStatus::complete;   // the predictor
    if (clouds_)   // CloudPredictorT (dust_cloud3d.cpp:1362-1436)
      return Check(dustb_cloud_pc2_predictor(&ctx_, pdrive->dt, 1, gpack_, stream_), "DepositDrag");
    return Check(dustb_pc2_predictor(&ctx_, pdrive->dt, 1, stream_), "DepositDrag");
  }
  if (clouds_) return Check(dustb_cloud_deposit_qp(&ctx_, a_dt(pdrive), 0.0, stream_), "DepositDrag");
  return Check(dustb_deposit_qp(&ctx_, a_dt(pdrive), 0.0, stream_), "DepositDrag");
}

TaskStatus DustGasDrag::RecvDepQP(Driver *pdrive, int stage) {
  if (!ctx_.phys.back_reaction) return TaskStatus::complete;
  if (coupling_ == DustCoupling::pc2 && stage != 1) return TaskStatus::complete;
  if (clouds_) return TaskStatus::complete;   // (the clouds deposit into the owner cells)
  if (refined_) return Check(dustb_ghost_add_plan(&ctx_, &plan_, ctx_.f.qdep, 5, stream_), "RecvDepQP");
  return Check(dustb_ghost_add(&ctx_, ctx_.f.qdep, 5, stream_), "RecvDepQP");
}

TaskStatus DustGasDrag::GasImplicitSolve(Driver *pdrive, int stage) {
  if (coupling_ == DustCoupling::pc2) {
    // the predictor's gas update with the stiffness record (UpdateStiffness, dust_pm.cpp:288-341)
    if (stage != 1 || !ctx_.phys.back_reaction) return TaskStatus::complete;
    return Check(dustb_pc2_apply_predictor(&ctx_, pdrive->dt, dev_scalars_ + 2, stream_),
                 "GasImplicitSolve");
  }
  TaskStatus ts = Check(dustb_solve_ustar(&ctx_, stream_), "GasImplicitSolve");
  if (ts != TaskStatus::complete || !ctx_.phys.back_reaction) return ts;
  // SolveCoupledStage (dust_solver.cpp:630-724): dc1 / dc2 defect-correction sweeps
  const int nsw = (ctx_.phys.drag_solver == DUSTB_SOLVER_DC2) ? 2
                : (ctx_.phys.drag_solver == DUSTB_SOLVER_DC1) ? 1 : 0;
  for (int w = 0; w < nsw && ts == TaskStatus::complete; ++w)
    ts = clouds_ ? Check(dustb_cloud_dc1_sweep(&ctx_, a_dt(pdrive), 0.0, gpack_, stream_),
                         "CloudDefectCorrection")
       : refined_ ? Check(dustb_dc1_sweep_plan(&ctx_, &plan_, a_dt(pdrive), coarse_,
                                               coarse_bytes_, stream_), "SolveCoupledStage")
                  : Check(dustb_dc1_sweep(&ctx_, a_dt(pdrive), 0.0, stream_), "SolveCoupledStage");
  return ts;
}

TaskStatus DustGasDrag::RecvUstar(Driver *pdrive, int stage) {
  if (coupling_ == DustCoupling::pc2) return TaskStatus::complete;   // (the midpoint covers ghosts)
  return CopyExchange(ctx_.f.ustar, 3, 1, "RecvUstar");
}

TaskStatus DustGasDrag::GatherKickPMBR(Driver *pdrive, int stage) {
  if (coupling_ == DustCoupling::pc2) return TaskStatus::complete;   // (inside the advance)
  if (clouds_)   // CloudGatherImplicit3D (dust_imex3d.cpp:181-308)
    return Check(dustb_cloud_gather_kick(&ctx_, a_dt(pdrive), 0.0, gpack_, stream_),
                 "GatherKickPMBR");
  return Check(dustb_gather_kick_pmbr(&ctx_, a_dt(pdrive), 0.0, stream_), "GatherKickPMBR");
}

TaskStatus DustGasDrag::RecvPMBR(Driver *pdrive, int stage) {
  if (!ctx_.phys.back_reaction) return TaskStatus::complete;
  if (coupling_ == DustCoupling::pc2 && stage != 2) return TaskStatus::complete;
  if (clouds_) return TaskStatus::complete;   // (the impulse went to the owner cells)
  if (refined_) return Check(dustb_ghost_add_plan(&ctx_, &plan_, ctx_.f.dmom, 3, stream_), "RecvPMBR");
  return Check(dustb_ghost_add(&ctx_, ctx_.f.dmom, 3, stream_), "RecvPMBR");
}

TaskStatus DustGasDrag::ApplyPMBR(Driver *pdrive, int stage) {
  if (!ctx_.phys.back_reaction) return TaskStatus::complete;
  if (coupling_ == DustCoupling::pc2) {
    if (stage != 2) return TaskStatus::complete;
    return Check(dustb_pc2_commit(&ctx_, 0.5, stream_), "ApplyPMBR");
  }
  if (clouds_) return Check(dustb_cloud_apply_pmbr(&ctx_, a_dt(pdrive), 0.0, stream_), "ApplyPMBR");
  return Check(dustb_apply_pmbr(&ctx_, a_dt(pdrive), stream_), "ApplyPMBR");
}

TaskStatus DustGasDrag::SetRefinableClouds(bool on) {
  if (on && !gpack_) {
    const long long bytes = dustb_cloud_gpack_bytes(&ctx_.mesh);
    if (bytes <= 0 || cudaMalloc(&gpack_, (size_t)bytes) != cudaSuccess) {
      gpack_ = nullptr;
      last_error_ = "SetRefinableClouds: gather pack not allocated";
      return TaskStatus::fail;
    }
  }
  clouds_ = on;
  return TaskStatus::complete;
}

TaskStatus DustGasDrag::RecvU(Driver *pdrive, int stage) {
  return CopyExchange(ctx_.f.u0, ctx_.f.nvar_gas, 0, "RecvU");
}

TaskStatus DustGasDrag::NewTimeStep(Driver *pdrive, int stage) {
  if (stage != pdrive->nexp_stages) return TaskStatus::complete;
  return Check(dustb_newdt(&ctx_, 1.0, dev_scalars_ + 3, stream_), "NewTimeStep");
}

TaskStatus DustGasDrag::SortParticles(double *spare_pr, int *spare_pi, void *scratch,
                                      long long bytes, int ncycle) {
  TaskStatus ts = Check(dustb_sort_by_cell(&ctx_, spare_pr, spare_pi, scratch, bytes, stream_),
                        "SortParticles");
  if (ts != TaskStatus::complete) return ts;
  // the sorted rows are the spares now (dust_cloud_device.cpp:1951-1954: swap)
  ctx_.part.pr = spare_pr;
  ctx_.part.pi = spare_pi;
  // after a sort in cell order the cloud order index is the identity (:1956-1975)
  if (cloud_order_interval_ > 0 && ncycle >= 0) {
    if ((ts = GrowCloudOrder()) != TaskStatus::complete) return ts;
    ts = Check(dustb_cloud_order_identity(&ctx_, cloud_ord_, cloud_ord_tag_, stream_),
               "SortParticles");
    if (ts != TaskStatus::complete) return ts;
    cloud_ord_n_ = ctx_.part.npart;
    cloud_sort_cycle_ = ncycle;
  }
  return ts;
}

TaskStatus DustGasDrag::DepositPointGravityDensity(double time, double *owned, double *halo) {
  dustb_ctx c = ctx_;
  c.mesh.time = time;
  return Check(dustb_point_gravity_density(&c, owned, halo, stream_), "DepositPointGravityDensity");
}

TaskStatus DustGasDrag::GatherPointGravityAcceleration(double time, const double *owned,
                                                       double *halo, double *acc,
                                                       long long acc_stride) {
  dustb_ctx c = ctx_;
  c.mesh.time = time;
  return Check(dustb_point_gravity_gather(&c, owned, halo, acc, acc_stride, stream_),
               "GatherPointGravityAcceleration");
}

TaskStatus DustGasDrag::DepositPointScienceFields(double time, double *out, double *halo,
                                                  bool mass_only, int species) {
  dustb_ctx c = ctx_;
  c.mesh.time = time;
  return Check(dustb_point_science_fields(&c, out, halo, mass_only ? 1 : 0, species, stream_),
               "DepositPointScienceFields");
}

// room for npart + npart/4 entries, as the reference allocates
TaskStatus DustGasDrag::GrowCloudOrder() {
  const int n = ctx_.part.npart;
  if (!dev_bad_ && cudaMalloc(&dev_bad_, sizeof(int)) != cudaSuccess) {
    dev_bad_ = nullptr;
    last_error_ = "UpdateCloudOrder: device counter not allocated";
    return TaskStatus::fail;
  }
  if (cloud_ord_cap_ >= n) return TaskStatus::complete;
  if (cloud_ord_) cudaFree(cloud_ord_);
  if (cloud_ord_tag_) cudaFree(cloud_ord_tag_);
  cloud_ord_ = nullptr;
  cloud_ord_tag_ = nullptr;
  cloud_ord_cap_ = 0;
  const int cap = n + n / 4;
  if (cudaMalloc(&cloud_ord_, sizeof(int) * (size_t)cap) != cudaSuccess ||
      cudaMalloc(&cloud_ord_tag_, sizeof(unsigned long long) * (size_t)cap) != cudaSuccess) {
    last_error_ = "UpdateCloudOrder: index not allocated";
    return TaskStatus::fail;
  }
  cloud_ord_cap_ = cap;
  return TaskStatus::complete;
}

TaskStatus DustGasDrag::UpdateCloudOrder(const Driver &drv, void *scratch, long long bytes) {
  if (cloud_order_interval_ <= 0) return TaskStatus::complete;
  const int npart = ctx_.part.npart;
  // the sort of this cycle left the identity index
  if (cloud_sort_cycle_ == drv.ncycle && cloud_ord_n_ == npart) return TaskStatus::complete;
  bool rebuild = (drv.ncycle % cloud_order_interval_ == 0) || cloud_ord_n_ == 0 ||
                 cloud_ord_n_ > npart;
  if (!rebuild) {
    TaskStatus ts = Check(dustb_cloud_order_check(&ctx_, cloud_ord_, cloud_ord_tag_,
                                                  cloud_ord_n_, dev_bad_, stream_),
                          "UpdateCloudOrder");
    if (ts != TaskStatus::complete) return ts;
    int bad = 0;
    if (cudaMemcpyAsync(&bad, dev_bad_, sizeof(int), cudaMemcpyDeviceToHost,
                        (cudaStream_t)stream_) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)stream_) != cudaSuccess) {
      last_error_ = "UpdateCloudOrder: check count not read";
      return TaskStatus::fail;
    }
    rebuild = bad > 0;
  }
  if (!rebuild) return TaskStatus::complete;
  if (npart < 2) { cloud_ord_n_ = 0; return TaskStatus::complete; }
  TaskStatus ts = GrowCloudOrder();
  if (ts != TaskStatus::complete) return ts;
  ts = Check(dustb_cloud_order(&ctx_, cloud_ord_, cloud_ord_tag_, scratch, bytes, stream_),
             "UpdateCloudOrder");
  if (ts != TaskStatus::complete) return ts;
  cloud_ord_n_ = npart;
  ++cloud_ord_builds_;
  return ts;
}

TaskStatus DustGasDrag::DoStage(Driver *pdrive, int stage) {
  // dust_tasks.cpp:56-107 on one rank, in dependency order: the register copy (pc2: the
  // midpoint), the gas update and the history term, the push and its migration, the deposit
  // and its exchange, the solve, the u* exchange, the gather-kick, its exchange and the
  // apply, the gas tail's exchange, the time step.  Each task is a no-op where the
  // reference's is for this coupling and stage.
  using Task = TaskStatus (DustGasDrag::*)(Driver *, int);
  static const Task order[] = {
      &DustGasDrag::FirstTwoImpRK,   &DustGasDrag::RKUpdate,       &DustGasDrag::AddDragHistoryGas,
      &DustGasDrag::ExplicitPush,    &DustGasDrag::UpdateParticleGIDs,
      &DustGasDrag::DepositDrag,     &DustGasDrag::RecvDepQP,      &DustGasDrag::GasImplicitSolve,
      &DustGasDrag::RecvUstar,       &DustGasDrag::GatherKickPMBR, &DustGasDrag::RecvPMBR,
      &DustGasDrag::ApplyPMBR,       &DustGasDrag::RecvU,          &DustGasDrag::NewTimeStep};
  for (Task t : order) {
    const TaskStatus ts = (this->*t)(pdrive, stage);
    if (ts != TaskStatus::complete) return ts;
  }
  return TaskStatus::complete;
}

TaskStatus DustGasDrag::DoCycle(Driver *pdrive) {
  for (int stage = 1; stage <= pdrive->nexp_stages; ++stage) {
    TaskStatus ts = DoStage(pdrive, stage);
    if (ts != TaskStatus::complete) return ts;
  }
  return TaskStatus::complete;
}

unsigned DustGasDrag::ErrorWord() {
  unsigned e = 0;
  cudaStreamSynchronize((cudaStream_t)stream_);
  cudaMemcpy(&e, ctx_.err, sizeof(unsigned), cudaMemcpyDeviceToHost);
  return e;
}

double DustGasDrag::NewDt() {
  double v = 0.0;
  cudaStreamSynchronize((cudaStream_t)stream_);
  cudaMemcpy(&v, dev_scalars_ + 3, sizeof(double), cudaMemcpyDeviceToHost);
  return v;
}

double DustGasDrag::ChiMax() {
  double v = 0.0;
  cudaStreamSynchronize((cudaStream_t)stream_);
  cudaMemcpy(&v, dev_scalars_ + 2, sizeof(double), cudaMemcpyDeviceToHost);
  return v;
}

void DustGasDrag::X3Removed(double out[2]) {
  cudaStreamSynchronize((cudaStream_t)stream_);
  cudaMemcpy(out, dev_scalars_, 2 * sizeof(double), cudaMemcpyDeviceToHost);
}

MixedDustGasDrag::MixedDustGasDrag(const dustb_ctx &ctx, void *stream, const double dx[3],
                                   int rows_per_tile, int chunk)
    : ctx_(ctx), stream_(stream) {
  std::memset(&mp_, 0, sizeof(mp_));
  for (int a = 0; a < 3; ++a) mp_.dx[a] = dx[a];
  mp_.rows_per_tile = rows_per_tile;
  mp_.chunk = chunk;
  tuned_ = rows_per_tile > 0 || chunk > 0;    // a given tile shape is kept
  ws_bytes_ = dustb_mixed_workspace_bytes(&ctx_.mesh, ctx_.part.npart);
  if (ws_bytes_ <= 0 || cudaMalloc(&ws_, (size_t)ws_bytes_) != cudaSuccess ||
      cudaMalloc(&dev_scalars_, 3 * sizeof(double)) != cudaSuccess) {
    last_error_ = "MixedDustGasDrag: workspace not allocated";
    return;
  }
  cudaMemsetAsync(dev_scalars_, 0, 3 * sizeof(double), (cudaStream_t)stream_);
  mp_.x3_removed = dev_scalars_;
}

MixedDustGasDrag::~MixedDustGasDrag() {
  if (ws_) cudaFree(ws_);
  if (dev_scalars_) cudaFree(dev_scalars_);
}

TaskStatus MixedDustGasDrag::Check(int rc, const char *what) {
  if (rc == DUSTB_OK) return TaskStatus::complete;
  last_error_ = std::string(what) + ": " + dustb_last_error() + " (" + std::to_string(rc) + ")";
  return TaskStatus::fail;
}

TaskStatus MixedDustGasDrag::Import() {
  return Check(dustb_mixed_import(&ctx_, &mp_, ws_, ws_bytes_, stream_), "mixed import");
}

TaskStatus MixedDustGasDrag::Export() {
  return Check(dustb_mixed_export(&ctx_, &mp_, ws_, ws_bytes_, stream_), "mixed export");
}

TaskStatus MixedDustGasDrag::Tune(double a_dt) {
  tuned_ = true;
  return Check(dustb_mixed_tune(&ctx_, &mp_, ws_, ws_bytes_, a_dt, nullptr, stream_),
               "mixed tune");
}

TaskStatus MixedDustGasDrag::ImexCycle(const Driver &drv) {
  if (!tuned_ && Tune(drv.gamma * drv.dt) != TaskStatus::complete) return TaskStatus::fail;
  dustb_imex_coeffs co;
  co.gamma = drv.gamma; co.dt = drv.dt; co.sh[0] = co.sh[1] = 0.0;
  ctx_.mesh.time = drv.time;
  return Check(dustb_mixed_imex_cycle(&ctx_, &mp_, ws_, ws_bytes_, &co, stream_), "mixed imex cycle");
}

TaskStatus MixedDustGasDrag::Pc2Cycle(const Driver &drv) {
  if (!tuned_ && Tune(0.5 * drv.dt) != TaskStatus::complete) return TaskStatus::fail;
  ctx_.mesh.time = drv.time;
  return Check(dustb_mixed_pc2_cycle(&ctx_, &mp_, ws_, ws_bytes_, drv.dt, dev_scalars_ + 2, stream_),
               "mixed pc2 cycle");
}

double MixedDustGasDrag::ChiMax() {
  double v = 0.0;
  cudaStreamSynchronize((cudaStream_t)stream_);
  cudaMemcpy(&v, dev_scalars_ + 2, sizeof(double), cudaMemcpyDeviceToHost);
  return v;
}

}  // namespace athenak_b200
