// refined_drag.cpp -- the C++ host layer (DustGasDrag) on a refined 3-D mesh: the case (mesh
// tables, the general deposit remap, the leaf tables, particles, gas) comes from a file that the
// Python test writes; the program copies it to the device, drives the task list the way the
// reference's host does (RefineClouds at the start of a cycle for clouds, then every stage's
// tasks), and writes the particle rows and the gas state back for the test to compare against
// the oracle.  Usage: refined_drag <case file> <result file>.  Exit status 0 when every task
// completed and no error bit is set.
//
// Case file: 24 int64 (nmb, nx1, nx2, nx3, ng, x3bc, npart, stride, nvar_gas, nseg, nent,
// nlev, nfine1..3, scheme, back_reaction, consistent_gas, drag_solver, clouds, split_enable,
// split_max_level, next_tag, ncycles), 12 doubles (x1min, x1max, x2min, x2max, x3min, x3max,
// dt, gamma, root_dx1..3, slack), then the arrays mb_size (nmb x 9 f64), nghbr (nmb x 27 i32),
// mb_lev (nmb i32), nghbr_ml (nmb x 56 i32), the plan (seg_tgt nseg, seg_ptr nseg + 1, ent_src
// nent i32, ent_w nent f64), the leaf tables (fbox nmb x 6, blev, nnb nmb, nb nmb x 64, nbs
// nmb x 64 x 3, nbmax nmb, safe nmb x 3 i32, lockey nmb i64, locblk nmb i32), pr (17 x stride
// f64), pi (5 x stride i32), u0 (nmb x nvar_gas x n3 x n2 x n1 f64).
// Result file: npart (int64), pr (17 x npart), pi (5 x npart), u0.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../athenak_b200/host/dust_gas_drag.hpp"

using athenak_b200::DustGasDrag;
using athenak_b200::Driver;
using athenak_b200::TaskStatus;

namespace {

template <typename T>
bool read_vec(FILE *f, std::vector<T> &v, size_t n) {
  v.resize(n);
  return n == 0 || fread(v.data(), sizeof(T), n, f) == n;
}

template <typename T>
T *to_device(const std::vector<T> &v) {
  T *d = nullptr;
  if (cudaMalloc(&d, (v.empty() ? 1 : v.size()) * sizeof(T)) != cudaSuccess) return nullptr;
  if (!v.empty()) cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return d;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: refined_drag <case> <result>\n");
    return 2;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) return 2;
  long long h[24];
  double r[12];
  if (fread(h, 8, 24, f) != 24 || fread(r, 8, 12, f) != 12) return 2;
  const int nmb = (int)h[0], nx1 = (int)h[1], nx2 = (int)h[2], nx3 = (int)h[3], ng = (int)h[4];
  const int npart = (int)h[6], nvg = (int)h[8], nseg = (int)h[9], nent = (int)h[10];
  const long long stride = h[7];
  const size_t cells = (size_t)(nx1 + 2 * ng) * (nx2 + 2 * ng) * (nx3 + 2 * ng);
  std::vector<double> mb, pw, pr, u0, ew;
  std::vector<int> nghbr, lev, nml, st, sp, es, fbox, blev, nnb, nb, nbs, nbmax, safe, locblk, pi;
  std::vector<long long> lockey;
  bool ok = read_vec(f, mb, (size_t)nmb * 9) && read_vec(f, nghbr, (size_t)nmb * 27) &&
            read_vec(f, lev, nmb) && read_vec(f, nml, (size_t)nmb * 56) &&
            read_vec(f, st, nseg) && read_vec(f, sp, (size_t)nseg + 1) && read_vec(f, es, nent) &&
            read_vec(f, ew, nent) && read_vec(f, fbox, (size_t)nmb * 6) && read_vec(f, blev, nmb) &&
            read_vec(f, nnb, nmb) && read_vec(f, nb, (size_t)nmb * 64) &&
            read_vec(f, nbs, (size_t)nmb * 64 * 3) && read_vec(f, nbmax, nmb) &&
            read_vec(f, safe, (size_t)nmb * 3) && read_vec(f, lockey, nmb) &&
            read_vec(f, locblk, nmb) && read_vec(f, pr, (size_t)17 * stride) &&
            read_vec(f, pi, (size_t)5 * stride) && read_vec(f, u0, (size_t)nmb * nvg * cells);
  fclose(f);
  if (!ok) {
    fprintf(stderr, "refined_drag: short case file\n");
    return 2;
  }
  dustb_ctx c;
  std::memset(&c, 0, sizeof(c));
  c.mesh.nmb = nmb; c.mesh.gids = 0;
  c.mesh.nx1 = nx1; c.mesh.nx2 = nx2; c.mesh.nx3 = nx3; c.mesh.ng = ng;
  c.mesh.multi_d = c.mesh.three_d = 1; c.mesh.x3bc = (int)h[5];
  c.mesh.x1min = r[0]; c.mesh.x1max = r[1]; c.mesh.x2min = r[2];
  c.mesh.x2max = r[3]; c.mesh.x3min = r[4]; c.mesh.x3max = r[5];
  c.mesh.mb_size = to_device(mb);
  c.mesh.nghbr = to_device(nghbr);
  c.mesh.mb_lev = to_device(lev);
  c.mesh.nghbr_ml = to_device(nml);
  c.part.pr = to_device(pr);
  c.part.pi = to_device(pi);
  c.part.stride = stride;
  c.part.npart = npart;
  const size_t fcell = (size_t)nmb * cells;
  c.f.u0 = to_device(u0);
  c.f.nvar_gas = nvg;
  std::vector<double> z4(fcell * nvg, 0.0), z5(fcell * 5, 0.0), z3(fcell * 3, 0.0);
  c.f.u1 = to_device(z4);
  c.f.qdep = to_device(z5);
  c.f.ustar = to_device(z3);
  c.f.dmom = to_device(z3);
  c.f.resid = to_device(std::vector<double>(fcell * 4, 0.0));
  c.f.work = to_device(z3);
  c.phys.scheme = (int)h[15];
  c.phys.back_reaction = (int)h[16];
  c.phys.consistent_gas = (int)h[17];
  c.phys.drag_solver = (int)h[18];
  c.phys.pc2_feedback_damping = 1;
  unsigned *err = nullptr;
  cudaMalloc(&err, sizeof(unsigned));
  cudaMemset(err, 0, sizeof(unsigned));
  c.err = err;
  // the plan and the leaf tables (their arrays on the device)
  dustb_dep_plan plan;
  plan.nseg = nseg;
  plan.seg_tgt = to_device(st);
  plan.seg_ptr = to_device(sp);
  plan.ent_src = to_device(es);
  plan.ent_w = to_device(ew);
  dustb_leaf_tables lt;
  std::memset(&lt, 0, sizeof(lt));
  lt.nlev = (int)h[11];
  for (int a = 0; a < 3; ++a) { lt.nfine[a] = (int)h[12 + a]; lt.root_dx[a] = r[8 + a]; }
  lt.fbox = to_device(fbox); lt.blev = to_device(blev); lt.nnb = to_device(nnb);
  lt.nb = to_device(nb); lt.nbs = to_device(nbs); lt.nbmax = to_device(nbmax);
  lt.safe = to_device(safe); lt.lockey = to_device(lockey); lt.locblk = to_device(locblk);

  cudaStream_t stream;
  cudaStreamCreate(&stream);
  DustGasDrag drag(c, stream);
  Driver drv;
  drv.SetImEx2PlusCoefficients(r[7]);
  drv.dt = r[6];
  const int clouds = (int)h[19];
  TaskStatus ts = drag.SetRefinedMesh(plan);
  void *scratch = nullptr;
  long long sbytes = 0;
  if (ts == TaskStatus::complete && clouds) {
    ts = drag.SetLeafTables(lt);
    dustb_cloud_split sp_ctl;
    std::memset(&sp_ctl, 0, sizeof(sp_ctl));
    // the split stops at cloud_split_max_level when that is set below the finest level
    sp_ctl.max_level = (h[21] >= 0 && h[21] < lt.nlev) ? (int)h[21] : lt.nlev;
    sp_ctl.split_everywhere = 0;
    sp_ctl.split_overlap = 1;
    sp_ctl.split_buffer = 0;
    sp_ctl.slack = r[11];
    drag.SetCloudSplit(sp_ctl, h[20] != 0, (int)h[21], (unsigned long long)h[22]);
    sbytes = dustb_cloud_split_scratch_bytes((int)stride);
    cudaMalloc(&scratch, (size_t)sbytes);
  }
  const int ncycles = (int)h[23];
  for (int cyc = 0; cyc < ncycles && ts == TaskStatus::complete; ++cyc) {
    if (clouds) ts = drag.RefineClouds(&drv, scratch, sbytes);
    if (ts == TaskStatus::complete) ts = drag.DoCycle(&drv);
    drv.time += drv.dt;
    ++drv.ncycle;
  }
  if (ts != TaskStatus::complete) {
    fprintf(stderr, "refined_drag: %s\n", drag.LastError().c_str());
    return 1;
  }
  const unsigned e = drag.ErrorWord();
  const int n = drag.Context().part.npart;
  std::vector<double> opr((size_t)17 * n), ou0(u0.size());
  std::vector<int> opi((size_t)5 * n);
  for (int q = 0; q < 17; ++q)
    cudaMemcpy(opr.data() + (size_t)q * n, c.part.pr + (size_t)q * stride, n * sizeof(double),
               cudaMemcpyDeviceToHost);
  for (int q = 0; q < 5; ++q)
    cudaMemcpy(opi.data() + (size_t)q * n, c.part.pi + (size_t)q * stride, n * sizeof(int),
               cudaMemcpyDeviceToHost);
  cudaMemcpy(ou0.data(), c.f.u0, ou0.size() * sizeof(double), cudaMemcpyDeviceToHost);
  FILE *o = fopen(argv[2], "wb");
  if (!o) return 2;
  const long long nn = n;
  fwrite(&nn, 8, 1, o);
  fwrite(opr.data(), 8, opr.size(), o);
  fwrite(opi.data(), 4, opi.size(), o);
  fwrite(ou0.data(), 8, ou0.size(), o);
  fclose(o);
  printf("refined_drag: npart %d, split pieces %d, switched %d, error word %u\n", n,
         drag.LastSplitPieces(), drag.LastSwitched(), e);
  return e == 0 ? 0 : 1;
}
