// pbin_tool.cpp -- writes particle science files (athenak_b200/host/pbin.hpp) for the tests.
//
//   pbin_tool host <dir>    seeded rows on the host, written by WritePbinFile (no GPU): the
//                           cases below, each as <dir>/<case>.pbin with its input rows in
//                           <dir>/<case>.rows (int64 n, int64 stride, then 17 x stride
//                           doubles and 5 x stride int32, the particle arrays as given)
//   pbin_tool device <dir>  rows seeded on the GPU (dustb_seed_uniform, some masses set to
//                           zero), written by WriteParticleBinary (versions 2 and 3)
//
// Exit status 0 when every file was written.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../athenak_b200/host/pbin.hpp"

using athenak_b200::PbinBlock;
using athenak_b200::PbinMeta;
using athenak_b200::PbinRows;

namespace {

constexpr int NB = 2, NX = 4;              // 2^3 blocks of 4^3 cells on [-0.5, 0.5)^3

std::vector<PbinBlock> blocks_of_mesh() {
  std::vector<PbinBlock> b;
  const double L = 1.0 / NB;
  for (int k = 0; k < NB; ++k)
    for (int j = 0; j < NB; ++j)
      for (int i = 0; i < NB; ++i) {
        PbinBlock x;
        x.gid = (k * NB + j) * NB + i;
        x.lx1 = i; x.lx2 = j; x.lx3 = k;
        x.x1min = -0.5 + i * L; x.x1max = x.x1min + L;
        x.x2min = -0.5 + j * L; x.x2max = x.x2min + L;
        x.x3min = -0.5 + k * L; x.x3max = x.x3min + L;
        b.push_back(x);
      }
  return b;
}

PbinMeta base_meta() {
  PbinMeta m;
  m.time = 1.25; m.dt = 0.01; m.cycle = 125; m.file_number = 3;
  m.basename = "dust_test"; m.source_commit = "test";
  m.nx1 = m.nx2 = m.nx3 = NB * NX; m.mb_nx1 = m.mb_nx2 = m.mb_nx3 = NX;
  m.x1min = m.x2min = m.x3min = -0.5; m.x1max = m.x2max = m.x3max = 0.5;
  m.input_dump = "<job>\nbasename = dust_test\n<dust>\ndeposit = tsc\n<par_end>\n";
  return m;
}

struct HostRows {
  int n = 0;
  std::vector<double> pr;
  std::vector<int> pi;
  double &r(int c, int p) { return pr[(size_t)c * n + p]; }
  int &i(int c, int p) { return pi[(size_t)c * n + p]; }
};

// a simple deterministic particle set: nsp species, some rows massless, tags with both words
HostRows make_rows(int n, int nsp, bool equal_mass, bool zero_some, double ts0) {
  HostRows h;
  h.n = n;
  h.pr.assign((size_t)17 * n, 0.0);
  h.pi.assign((size_t)5 * n, 0);
  for (int p = 0; p < n; ++p) {
    const double a = std::sin(0.37 * p + 0.1), b = std::cos(0.91 * p), c = std::sin(1.7 * p + 2.0);
    h.r(0, p) = 0.49 * a; h.r(2, p) = 0.49 * b; h.r(4, p) = 0.49 * c;
    h.r(1, p) = 0.01 * b; h.r(3, p) = -0.02 * c; h.r(5, p) = 0.03 * a;
    const int s = p % nsp;
    h.r(15, p) = (nsp == 1) ? ts0 : 0.01 * (s + 1);
    h.r(16, p) = equal_mass ? 1.0 / 1024 : (1.0 + 0.5 * s + 1e-3 * p) / 1024;
    if (zero_some && p % 7 == 3) h.r(16, p) = 0.0;
    h.i(0, p) = 0;                                        // PGID
    h.i(1, p) = (p % 5 == 0) ? -1 - p : p;                // PTAG (negative low words too)
    h.i(2, p) = s;                                        // PSP
    h.i(4, p) = (p % 3 == 0) ? 1 : 0;                     // PTAGH
  }
  return h;
}

dustb_pbin_stats stats_of(HostRows &h, double ts0) {
  dustb_pbin_stats s{};
  s.mass_min = 1.7976931348623157e308; s.mass_max = -1.7976931348623157e308;
  for (int p = 0; p < h.n; ++p) {
    const double m = h.r(16, p);
    if (m == 0.0) { ++s.zero_mass_rows; continue; }
    ++s.active_rows;
    if (!(m > 0.0) || !std::isfinite(m)) ++s.invalid_mass_rows;
    if (h.i(4, p) < 0) ++s.negative_tag_rows;
    if (h.i(2, p) != 0 || h.r(15, p) != ts0) ++s.differ_rows;
    s.mass_min = std::fmin(s.mass_min, m); s.mass_max = std::fmax(s.mass_max, m);
  }
  return s;
}

bool save_rows(const std::string &path, HostRows &h) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const long long hdr[2] = {h.n, h.n};
  bool ok = std::fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
            std::fwrite(h.pr.data(), sizeof(double), h.pr.size(), f) == h.pr.size() &&
            std::fwrite(h.pi.data(), sizeof(int), h.pi.size(), f) == h.pi.size();
  return std::fclose(f) == 0 && ok;
}

// the host columns of the active rows
PbinRows host_rows(HostRows &h, std::uint64_t nact) {
  PbinRows r;
  r.n = nact;
  r.fetch = [&h](int column, std::uint64_t itemsize, std::vector<unsigned char> &out) {
    std::vector<unsigned char> tmp;
    for (int p = 0; p < h.n; ++p) {
      if (h.r(16, p) == 0.0) continue;
      unsigned char v[8];
      if (column == DUSTB_PBIN_ID) {
        const std::uint64_t t = ((std::uint64_t)(std::uint32_t)h.i(4, p) << 32) |
                                (std::uint32_t)h.i(1, p);
        std::memcpy(v, &t, 8);
      } else if (column == DUSTB_PBIN_SPECIES) {
        const std::uint32_t s = (std::uint32_t)h.i(2, p);
        std::memcpy(v, &s, 4);
      } else {
        static const int row[10] = {0, 0, 0, 2, 4, 1, 3, 5, 16, 15};
        const double x = h.r(row[column], p);
        if (itemsize == 4) { const float y = (float)x; std::memcpy(v, &y, 4); }
        else std::memcpy(v, &x, 8);
      }
      tmp.insert(tmp.end(), v, v + itemsize);
    }
    out.swap(tmp);
    return true;
  };
  return r;
}

int host_cases(const std::string &dir) {
  struct Case { const char *name; int n, nsp; bool equal_mass, zero_some, single, compress; std::uint64_t chunk; };
  const Case cases[] = {
      {"two_species", 3000, 2, false, true, false, false, 0},
      {"one_species_constants", 2000, 1, true, true, false, false, 0},
      {"single_precision", 1500, 3, false, false, true, false, 0},
      {"compressed", 5000, 2, false, true, false, true, 1000},
      {"compressed_single", 2500, 1, true, false, true, true, 700},
      {"empty", 0, 1, true, false, false, true, 1000},
  };
  const double ts0 = 0.1;
  int bad = 0;
  for (const auto &c : cases) {
    if (c.compress && !athenak_b200::PbinCanCompress()) {
      std::printf("%s: skipped (no zlib)\n", c.name);
      continue;
    }
    HostRows h = make_rows(c.n, c.nsp, c.equal_mass, c.zero_some, ts0);
    PbinMeta m = base_meta();
    m.nspecies = c.nsp;
    for (int s = 0; s < c.nsp; ++s) m.taus.push_back(c.nsp == 1 ? ts0 : 0.01 * (s + 1));
    m.single_precision = c.single;
    m.compress = c.compress;
    if (c.chunk) m.chunk_rows = c.chunk;
    m.shearing_box = (c.nsp == 2);
    const dustb_pbin_stats st = stats_of(h, ts0);
    const std::string path = dir + "/" + c.name + ".pbin";
    const std::string err = athenak_b200::WritePbinFile(path, m, st, host_rows(h, st.active_rows),
                                                        blocks_of_mesh());
    if (!err.empty() || !save_rows(dir + "/" + c.name + ".rows", h)) {
      std::printf("%s: %s\n", c.name, err.c_str());
      ++bad;
    } else {
      std::printf("%s: written, %lld rows\n", c.name, st.active_rows);
    }
  }
  return bad;
}

int device_cases(const std::string &dir) {
  // a periodic 8^3 mesh of 2^3 blocks seeded on the device
  const int nmb = NB * NB * NB, ppc = 2, nsp = 2;
  const int npart = nmb * NX * NX * NX * ppc * nsp;
  std::vector<PbinBlock> blocks = blocks_of_mesh();
  std::vector<double> mb((size_t)nmb * 9);
  for (int m = 0; m < nmb; ++m) {
    const PbinBlock &b = blocks[m];
    const double v[9] = {b.x1min, b.x2min, b.x3min, b.x1max, b.x2max, b.x3max,
                         (b.x1max - b.x1min) / NX, (b.x2max - b.x2min) / NX, (b.x3max - b.x3min) / NX};
    std::memcpy(&mb[(size_t)m * 9], v, sizeof(v));
  }
  double *d_pr = nullptr, *d_mb = nullptr, *d_u0 = nullptr;
  int *d_pi = nullptr;
  unsigned *d_err = nullptr;
  const int n1 = NX + 4;
  const size_t cells = (size_t)nmb * 4 * n1 * n1 * n1;
  if (cudaMalloc(&d_pr, sizeof(double) * 17 * npart) != cudaSuccess ||
      cudaMalloc(&d_pi, sizeof(int) * 5 * npart) != cudaSuccess ||
      cudaMalloc(&d_mb, sizeof(double) * mb.size()) != cudaSuccess ||
      cudaMalloc(&d_u0, sizeof(double) * cells) != cudaSuccess ||
      cudaMalloc(&d_err, sizeof(unsigned)) != cudaSuccess) {
    std::printf("device: allocation failed\n");
    return 1;
  }
  cudaMemcpy(d_mb, mb.data(), sizeof(double) * mb.size(), cudaMemcpyHostToDevice);
  cudaMemset(d_u0, 0, sizeof(double) * cells);
  cudaMemset(d_err, 0, sizeof(unsigned));
  dustb_ctx c;
  std::memset(&c, 0, sizeof(c));
  c.mesh.nmb = nmb; c.mesh.nx1 = c.mesh.nx2 = c.mesh.nx3 = NX; c.mesh.ng = 2;
  c.mesh.multi_d = c.mesh.three_d = 1;
  c.mesh.x1min = c.mesh.x2min = c.mesh.x3min = -0.5;
  c.mesh.x1max = c.mesh.x2max = c.mesh.x3max = 0.5;
  c.mesh.mb_size = d_mb;
  c.part.pr = d_pr; c.part.pi = d_pi; c.part.stride = npart; c.part.npart = npart;
  c.f.u0 = d_u0; c.f.nvar_gas = 4;
  c.phys.scheme = DUSTB_TSC;
  c.err = d_err;
  dustb_seed_desc sd;
  std::memset(&sd, 0, sizeof(sd));
  sd.seed = 5; sd.nspecies = nsp;
  for (int s = 0; s < nsp; ++s) {
    sd.ppc[s] = ppc; sd.taus[s] = 0.1 * (s + 1); sd.mass[s] = 1e-3 * (s + 1);
    sd.vx[s] = 0.01; sd.vy[s] = -0.02; sd.vz[s] = 0.0;
  }
  sd.vel_noise = 0.01; sd.rho0 = 1.0; sd.nb1 = sd.nb2 = sd.nb3 = NB;
  int bad = 0;
  if (dustb_seed_uniform(&c, &sd, nullptr) != DUSTB_OK) { std::printf("device: seed failed\n"); return 1; }
  // every 11th row massless (left out), a tag with a high word
  for (int p = 3; p < npart; p += 11) {
    const double z = 0.0;
    cudaMemcpy(d_pr + (size_t)16 * npart + p, &z, sizeof(double), cudaMemcpyHostToDevice);
  }
  const int hi = 7;
  cudaMemcpy(d_pi + (size_t)4 * npart + 2, &hi, sizeof(int), cudaMemcpyHostToDevice);
  cudaDeviceSynchronize();
  HostRows h;
  h.n = npart;
  h.pr.resize((size_t)17 * npart);
  h.pi.resize((size_t)5 * npart);
  cudaMemcpy(h.pr.data(), d_pr, sizeof(double) * h.pr.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(h.pi.data(), d_pi, sizeof(int) * h.pi.size(), cudaMemcpyDeviceToHost);
  for (int v = 0; v < 3; ++v) {
    if (v == 2 && !athenak_b200::PbinCanCompress()) continue;
    PbinMeta m = base_meta();
    m.nspecies = nsp;
    m.taus = {0.1, 0.2};
    m.single_precision = (v == 1);
    m.compress = (v == 2);
    m.chunk_rows = 1500;
    const char *name = v == 0 ? "device_v2" : (v == 1 ? "device_v2_single" : "device_v3");
    dustb_pbin_stats st{};
    const std::string err = athenak_b200::WriteParticleBinary(c, nullptr, dir + "/" + name + ".pbin",
                                                              m, blocks, &st);
    if (!err.empty() || !save_rows(dir + "/" + name + ".rows", h)) {
      std::printf("%s: %s\n", name, err.c_str());
      ++bad;
    } else {
      std::printf("%s: written, %lld rows, %lld massless left out\n", name, st.active_rows,
                  st.zero_mass_rows);
    }
  }
  cudaFree(d_pr); cudaFree(d_pi); cudaFree(d_mb); cudaFree(d_u0); cudaFree(d_err);
  return bad;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::printf("usage: pbin_tool host|device <dir>\n");
    return 2;
  }
  const std::string mode = argv[1], dir = argv[2];
  const int bad = (mode == "host") ? host_cases(dir) : device_cases(dir);
  return bad ? 1 : 0;
}
