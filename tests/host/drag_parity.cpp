// drag_parity.cpp -- the drag step driven the way the reference's host drives it: the
// DustGasDrag task functions of the C++ host layer (athenak_b200/host/dust_gas_drag.hpp), one
// stage after another in the task list's order, on the GPU; the CPU oracle (test
// infrastructure, oracle/dust_oracle.c) runs the same cycles on a host copy of the same
// seeded inputs.  imex2+/dc2 and pc2 on a periodic 16^3 mesh of 8^3 MeshBlocks (a 3-D shearing
// box: rotation, shear drift): positions within 1e-12 of the box, velocities within 1e-12 of
// their scale, the gas momentum within 1e-11 of its scale, PGID identical, no error bit;
// then the same cycles in the mixed-precision form (MixedDustGasDrag) at its tolerance.
// After the FP64 imex2+ cycles the cloud order index (UpdateCloudOrder) runs through its
// control on the moved rows.  Exit status 0 on agreement.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../athenak_b200/host/dust_gas_drag.hpp"

extern "C" {
unsigned oracle_imex_cycle(const dustb_ctx *c, double gamma, double dt, const double sh[2],
                           double *x3_removed);
unsigned oracle_pc2_cycle(const dustb_ctx *c, double dt, double *chi_out, double *x3_removed);
unsigned oracle_cloud_imex_cycle(const dustb_ctx *c, double gamma, double dt, const double sh[2],
                                 double *x3_removed);
unsigned oracle_cloud_pc2_cycle(const dustb_ctx *c, double dt, double *chi_out, double *x3_removed);
void oracle_ghost_copy(const dustb_ctx *c, double *a, int nvar, int x3_bcs);
void oracle_set_threads(int n);
void oracle_cloud_order(const dustb_ctx *c, int *ord, uint64_t *tag);
}

namespace {

constexpr int NX = 8, NB = 2, NG = 2, N1 = NX + 2 * NG;
constexpr double LO = -0.05, HI = 0.05;

struct Arrays {               // one set of the pack's arrays (host or device)
  double *pr, *u0, *u1, *qdep, *ustar, *dmom, *resid, *work, *mb;
  int *pi, *nghbr, *sbgid;
  unsigned *err;
};

const int NMB = NB * NB * NB;
const size_t CELLS = (size_t)N1 * N1 * N1;

int dir(int o1, int o2, int o3) { return (o3 + 1) * 9 + (o2 + 1) * 3 + (o1 + 1); }

// the uniform periodic mesh: RegionSize of each block and the same-level neighbour gids
void mesh_tables(std::vector<double> &mb, std::vector<int> &ng) {
  mb.assign(NMB * 9, 0.0);
  ng.assign(NMB * 27, -1);
  const double L = (HI - LO) / NB;
  for (int b3 = 0; b3 < NB; ++b3)
    for (int b2 = 0; b2 < NB; ++b2)
      for (int b1 = 0; b1 < NB; ++b1) {
        const int m = (b3 * NB + b2) * NB + b1;
        const int b[3] = {b1, b2, b3};
        for (int a = 0; a < 3; ++a) {
          mb[m * 9 + a] = LO + b[a] * L;
          mb[m * 9 + 3 + a] = LO + (b[a] + 1) * L;
          mb[m * 9 + 6 + a] = L / NX;
        }
        for (int o3 = -1; o3 <= 1; ++o3)
          for (int o2 = -1; o2 <= 1; ++o2)
            for (int o1 = -1; o1 <= 1; ++o1) {
              if (!o1 && !o2 && !o3) continue;
              const int t1 = (b1 + o1 + NB) % NB, t2 = (b2 + o2 + NB) % NB, t3 = (b3 + o3 + NB) % NB;
              ng[m * 27 + dir(o1, o2, o3)] = (t3 * NB + t2) * NB + t1;
            }
      }
}

dustb_ctx make_ctx(const Arrays &a, int npart) {
  dustb_ctx c;
  std::memset(&c, 0, sizeof(c));
  c.mesh.nmb = NMB; c.mesh.gids = 0;
  c.mesh.nx1 = c.mesh.nx2 = c.mesh.nx3 = NX; c.mesh.ng = NG;
  c.mesh.multi_d = c.mesh.three_d = 1; c.mesh.x3bc = DUSTB_X3_PERIODIC;
  c.mesh.x1min = c.mesh.x2min = c.mesh.x3min = LO;
  c.mesh.x1max = c.mesh.x2max = c.mesh.x3max = HI;
  c.mesh.mb_size = a.mb; c.mesh.nghbr = a.nghbr;
  c.mesh.sb_gid = a.sbgid;
  c.part.pr = a.pr; c.part.pi = a.pi; c.part.stride = npart; c.part.npart = npart;
  c.f.u0 = a.u0; c.f.u1 = a.u1; c.f.nvar_gas = 4; c.f.qdep = a.qdep; c.f.ustar = a.ustar;
  c.f.dmom = a.dmom; c.f.resid = a.resid; c.f.work = a.work;
  c.phys.scheme = DUSTB_TSC; c.phys.back_reaction = 1; c.phys.consistent_gas = 1;
  c.phys.drag_solver = DUSTB_SOLVER_DC2; c.phys.shearing_box = 1; c.phys.stratified = 0;
  c.phys.pc2_feedback_damping = 1; c.phys.qshear = 1.5; c.phys.omega0 = 1.0;
  c.err = a.err;
  return c;
}

const size_t NF[8] = {4, 4, 5, 3, 3, 4, 3};   // u0 u1 qdep ustar dmom resid work

// UpdateCloudOrder's control on the pack's rows (cloud_order_interval = 4): the first build
// equals the oracle's index of the same rows (slots and tags bit-exact); a passing check at
// the next cycle keeps it; a sort at cycle 3 leaves the identity, which that cycle keeps; the
// rebuild at the interval (cycle 4) gives the identity again on the sorted rows; a tag
// changed under the index fails the next check and the rebuilt index holds the new tag.
// The sort moves the rows into spares this function allocates and frees: call it last.
bool cloud_order_checks(athenak_b200::DustGasDrag &drag, int npart, std::vector<double> &mb,
                        std::vector<int> &ng) {
  using athenak_b200::TaskStatus;
  athenak_b200::Driver drv;
  const long long bytes = dustb_sort_scratch_bytes(&drag.Context().mesh, npart);
  void *scratch = nullptr;
  double *spr = nullptr;
  int *spi = nullptr;
  cudaMalloc(&scratch, (size_t)bytes);
  cudaMalloc(&spr, sizeof(double) * 17 * npart);
  cudaMalloc(&spi, sizeof(int) * 5 * npart);
  std::vector<int> go(npart);
  std::vector<unsigned long long> gt(npart);
  auto index = [&]() {
    cudaMemcpy(go.data(), drag.CloudOrder(), sizeof(int) * npart, cudaMemcpyDeviceToHost);
    cudaMemcpy(gt.data(), drag.CloudOrderTags(), sizeof(unsigned long long) * npart,
               cudaMemcpyDeviceToHost);
  };
  auto identity = [&]() {
    index();
    bool id = true;
    for (int k = 0; k < npart; ++k) id = id && go[k] == k;
    return id;
  };
  auto update = [&](int cyc) {
    drv.ncycle = cyc;
    return drag.UpdateCloudOrder(drv, scratch, bytes) == TaskStatus::complete;
  };
  drag.SetCloudOrderInterval(4);
  bool ok = update(1) && drag.CloudOrderBuilds() == 1 && drag.CloudOrderLength() == npart;
  // the oracle's index of the same rows
  std::vector<double> hpr(17 * (size_t)npart);
  std::vector<int> hpi(5 * (size_t)npart);
  cudaMemcpy(hpr.data(), drag.Context().part.pr, sizeof(double) * hpr.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(hpi.data(), drag.Context().part.pi, sizeof(int) * hpi.size(), cudaMemcpyDeviceToHost);
  Arrays h{hpr.data(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, mb.data(),
           hpi.data(), ng.data(), nullptr, nullptr};
  dustb_ctx hc = make_ctx(h, npart);
  std::vector<int> oo(npart);
  std::vector<uint64_t> ot(npart);
  oracle_cloud_order(&hc, oo.data(), ot.data());
  index();
  bool same = true, moved = false;
  for (int k = 0; k < npart; ++k) {
    same = same && go[k] == oo[k] && gt[k] == (unsigned long long)ot[k];
    moved = moved || go[k] != k;
  }
  ok = ok && same && moved;
  ok = ok && update(2) && drag.CloudOrderBuilds() == 1;
  ok = ok && drag.SortParticles(spr, spi, scratch, bytes, 3) == TaskStatus::complete;
  ok = ok && update(3) && drag.CloudOrderBuilds() == 1 && identity();
  ok = ok && update(4) && drag.CloudOrderBuilds() == 2 && identity();
  // a new tag in slot 5 (PTAG row)
  const int newtag = 987654321;
  cudaMemcpy(drag.Context().part.pi + 1 * (size_t)npart + 5, &newtag, sizeof(int),
             cudaMemcpyHostToDevice);
  ok = ok && update(5) && drag.CloudOrderBuilds() == 3 && identity() &&
       (unsigned)(gt[5] & 0xffffffffull) == (unsigned)newtag;
  std::printf("cloud order index: builds %d, length %d, first build %s the oracle's: %s\n",
              drag.CloudOrderBuilds(), drag.CloudOrderLength(), same ? "equals" : "DIFFERS FROM",
              ok ? "ok" : "MISMATCH");
  cudaFree(scratch);
  cudaFree(spr);
  cudaFree(spi);
  return ok;
}

// mixed: the mixed-precision form (MixedDustGasDrag) against the oracle at the mixed form's
// stated tolerance (velocities 1e-5 of their scale, positions 1e-5 of a cell, the gas
// momentum 1e-5 of its scale); the gas ghost cells first take the copy exchange the mixed
// form reads through the owning blocks
int run(athenak_b200::DustCoupling coupling, const char *name, bool mixed = false,
        bool clouds = false) {
  const int ppc = 2, nsp = 2;
  const int npart = NMB * NX * NX * NX * ppc * nsp;
  std::vector<double> mb; std::vector<int> ng;
  mesh_tables(mb, ng);
  std::vector<int> sbgid(2 * NB * NB, 0);
  // device arrays
  Arrays d{};
  double **fd[7] = {&d.u0, &d.u1, &d.qdep, &d.ustar, &d.dmom, &d.resid, &d.work};
  cudaMalloc(&d.pr, sizeof(double) * 17 * npart);
  cudaMalloc(&d.pi, sizeof(int) * 5 * npart);
  for (int f = 0; f < 7; ++f) {
    cudaMalloc(fd[f], sizeof(double) * NMB * NF[f] * CELLS);
    cudaMemset(*fd[f], 0, sizeof(double) * NMB * NF[f] * CELLS);
  }
  cudaMalloc(&d.mb, sizeof(double) * mb.size());
  cudaMalloc(&d.nghbr, sizeof(int) * ng.size());
  cudaMalloc(&d.sbgid, sizeof(int) * sbgid.size());
  cudaMalloc(&d.err, sizeof(unsigned));
  cudaMemcpy(d.mb, mb.data(), sizeof(double) * mb.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d.nghbr, ng.data(), sizeof(int) * ng.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d.sbgid, sbgid.data(), sizeof(int) * sbgid.size(), cudaMemcpyHostToDevice);
  cudaMemset(d.err, 0, sizeof(unsigned));
  dustb_ctx dc = make_ctx(d, npart);
  // seeded inputs (the NSH-like drift of two species plus noise)
  dustb_seed_desc sd;
  std::memset(&sd, 0, sizeof(sd));
  sd.seed = 11; sd.nspecies = nsp;
  const double vol = std::pow(HI - LO, 3.0);
  const double taus[2] = {0.01, 0.3}, eps[2] = {0.5, 1.0};
  for (int s = 0; s < nsp; ++s) {
    sd.ppc[s] = ppc; sd.taus[s] = taus[s];
    sd.mass[s] = eps[s] * vol / (NMB * NX * NX * NX * ppc);
    sd.vx[s] = -0.02 * (s + 1); sd.vy[s] = -0.03; sd.vz[s] = 0.0;
  }
  sd.vel_noise = 0.02; sd.rho0 = 1.0; sd.ug[0] = 0.01; sd.ug[1] = -0.04; sd.gas_noise = 1e-2;
  sd.nb1 = sd.nb2 = sd.nb3 = NB;
  if (dustb_seed_uniform(&dc, &sd, nullptr) != DUSTB_OK) { std::printf("%s: seed failed\n", name); return 1; }
  cudaDeviceSynchronize();
  // the oracle's host copy
  std::vector<double> hpr(17 * (size_t)npart), hf[7];
  std::vector<int> hpi(5 * (size_t)npart);
  cudaMemcpy(hpr.data(), d.pr, sizeof(double) * hpr.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(hpi.data(), d.pi, sizeof(int) * hpi.size(), cudaMemcpyDeviceToHost);
  double *hptr[7];
  for (int f = 0; f < 7; ++f) {
    hf[f].assign(NMB * NF[f] * CELLS, 0.0);
    cudaMemcpy(hf[f].data(), *fd[f], sizeof(double) * hf[f].size(), cudaMemcpyDeviceToHost);
    hptr[f] = hf[f].data();
  }
  unsigned herr = 0;
  Arrays h{hpr.data(), hptr[0], hptr[1], hptr[2], hptr[3], hptr[4], hptr[5], hptr[6], mb.data(),
           hpi.data(), ng.data(), sbgid.data(), &herr};
  dustb_ctx hc = make_ctx(h, npart);
  // three cycles each way
  athenak_b200::Driver drv;
  drv.SetImEx2PlusCoefficients(1.0 + 1.0 / std::sqrt(2.0));
  drv.dt = 2e-3;
  athenak_b200::DustGasDrag drag(dc, nullptr, coupling);
  if (clouds) {
    // refinable clouds of levels 0-3 on a periodic box (the shearing box's push terms kept,
    // its faces plain periodic here)
    std::vector<int> lev(npart);
    for (int p = 0; p < npart; ++p) lev[p] = p % 4;
    cudaMemcpy(d.pi + (size_t)3 * npart, lev.data(), sizeof(int) * npart, cudaMemcpyHostToDevice);
    std::memcpy(hpi.data() + (size_t)3 * npart, lev.data(), sizeof(int) * npart);
    if (drag.SetRefinableClouds(true) != athenak_b200::TaskStatus::complete) {
      std::printf("%s: %s\n", name, drag.LastError().c_str());
      return 1;
    }
  }
  const double sh[2] = {0.0, 0.0};
  double x3o[2] = {0.0, 0.0}, chi = 0.0;
  unsigned oerr = 0;
  const double cell[3] = {(HI - LO) / (NB * NX), (HI - LO) / (NB * NX), (HI - LO) / (NB * NX)};
  athenak_b200::MixedDustGasDrag mx(dc, nullptr, cell);
  if (mixed) {
    dustb_ghost_copy(&dc, d.u0, 4, 0, nullptr);
    oracle_ghost_copy(&hc, hf[0].data(), 4, 0);
    if (mx.Import() != athenak_b200::TaskStatus::complete) {
      std::printf("%s: %s\n", name, mx.LastError().c_str());
      return 1;
    }
  }
  for (int cyc = 0; cyc < 3; ++cyc) {
    athenak_b200::TaskStatus ts;
    if (!mixed) ts = drag.DoCycle(&drv);
    else if (coupling == athenak_b200::DustCoupling::imex) ts = mx.ImexCycle(drv);
    else ts = mx.Pc2Cycle(drv);
    if (ts != athenak_b200::TaskStatus::complete) {
      std::printf("%s: task failed: %s%s\n", name, drag.LastError().c_str(), mx.LastError().c_str());
      return 1;
    }
    oerr |= clouds ? ((coupling == athenak_b200::DustCoupling::imex)
                          ? oracle_cloud_imex_cycle(&hc, drv.gamma, drv.dt, sh, x3o)
                          : oracle_cloud_pc2_cycle(&hc, drv.dt, &chi, x3o))
            : (coupling == athenak_b200::DustCoupling::imex)
                ? oracle_imex_cycle(&hc, drv.gamma, drv.dt, sh, x3o)
                : oracle_pc2_cycle(&hc, drv.dt, &chi, x3o);
  }
  if (mixed && mx.Export() != athenak_b200::TaskStatus::complete) {
    std::printf("%s: %s\n", name, mx.LastError().c_str());
    return 1;
  }
  const unsigned gerr = drag.ErrorWord();
  std::vector<double> gpr(hpr.size()), gu0(hf[0].size());
  std::vector<int> gpi(hpi.size());
  cudaMemcpy(gpr.data(), drag.Context().part.pr, sizeof(double) * gpr.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(gpi.data(), drag.Context().part.pi, sizeof(int) * gpi.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(gu0.data(), d.u0, sizeof(double) * gu0.size(), cudaMemcpyDeviceToHost);
  double dx = 0.0, dv = 0.0, vs = 0.0, du = 0.0, us = 0.0;
  for (int p = 0; p < npart; ++p)
    for (int r = 0; r < 6; ++r) {
      const double a = gpr[(size_t)r * npart + p], b = hpr[(size_t)r * npart + p];
      if (r % 2 == 0) dx = std::fmax(dx, std::fabs(a - b));
      else { dv = std::fmax(dv, std::fabs(a - b)); vs = std::fmax(vs, std::fabs(b)); }
    }
  for (size_t q = 0; q < gu0.size(); ++q) {
    du = std::fmax(du, std::fabs(gu0[q] - hf[0][q]));
    us = std::fmax(us, std::fabs(hf[0][q]));
  }
  bool pgid = true;
  for (int p = 0; p < npart; ++p) pgid = pgid && gpi[p] == hpi[p];
  const double tp = mixed ? 1e-5 * cell[0] : 1e-12 * (HI - LO), tv = mixed ? 1e-5 : 1e-12;
  const double tu = mixed ? 1e-5 : 1e-11;
  const bool ok = gerr == 0 && oerr == 0 && pgid && dx <= tp && dv <= tv * vs && du <= tu * us;
  std::printf("%s: particles %d, max |dx| %.3e, max |dv| %.3e (scale %.3e), max |du0| %.3e "
              "(scale %.3e), PGID %s, error words %u/%u: %s\n",
              name, npart, dx, dv, vs, du, us, pgid ? "identical" : "DIFFER", gerr, oerr,
              ok ? "ok" : "MISMATCH");
  const bool cord = mixed || clouds || coupling != athenak_b200::DustCoupling::imex ||
                    cloud_order_checks(drag, npart, mb, ng);
  for (int f = 0; f < 7; ++f) cudaFree(*fd[f]);
  cudaFree(d.pr); cudaFree(d.pi); cudaFree(d.mb); cudaFree(d.nghbr); cudaFree(d.sbgid);
  cudaFree(d.err);
  return ok && cord ? 0 : 1;
}

}  // namespace

int main() {
  oracle_set_threads(1);
  int bad = 0;
  bad += run(athenak_b200::DustCoupling::imex, "imex2+/dc2 cycles");
  bad += run(athenak_b200::DustCoupling::pc2, "pc2 cycles");
  bad += run(athenak_b200::DustCoupling::imex, "mixed imex2+/dc2 cycles", true);
  bad += run(athenak_b200::DustCoupling::pc2, "mixed pc2 cycles", true);
  bad += run(athenak_b200::DustCoupling::imex, "refinable-cloud imex2+/dc2 cycles", false, true);
  bad += run(athenak_b200::DustCoupling::pc2, "refinable-cloud pc2 cycles", false, true);
  return bad ? 1 : 0;
}
