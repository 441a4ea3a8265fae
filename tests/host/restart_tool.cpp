// restart_tool.cpp -- the particle section of the restart file (athenak_b200/host/restart.hpp)
// for the tests.
//
//   restart_tool host <dir>    host rows: a section written and parsed back (rows and records
//                              bit for bit), a version-1 section built here byte by byte and
//                              parsed (the high tag words 0, the int32 counter), and damaged
//                              sections rejected; writes <dir>/host.rst and <dir>/host.rows
//   restart_tool ranks <dir>   a file of two ranks' sections: split, each rank's own section
//                              taken back exactly, the particles of other block layouts
//                              gathered from every section, damaged files rejected; writes
//                              <dir>/ranks.rst (the two sections)
//   restart_tool device <dir>  rows seeded on the GPU, packed from the device, restored into
//                              arrays of another capacity and compared bit for bit
//
// Prints one line per check; exit status 0 when all pass.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../athenak_b200/host/restart.hpp"

using athenak_b200::ParticleRestartSection;
using athenak_b200::ParticleRestartState;

namespace {

int bad = 0;
void check(bool ok, const char *what) {
  std::printf("%s: %s\n", what, ok ? "ok" : "FAILED");
  if (!ok) ++bad;
}

void make_rows(int n, long long stride, std::vector<double> &pr, std::vector<int> &pi) {
  pr.assign((std::size_t)17 * stride, -7.0);   // the capacity tail holds other values
  pi.assign((std::size_t)5 * stride, -9);
  for (int p = 0; p < n; ++p) {
    for (int r = 0; r < 17; ++r) pr[(std::size_t)r * stride + p] = std::sin(0.1 * p + r) * (r + 1);
    pi[p] = p % 8;                                   // PGID
    pi[(std::size_t)1 * stride + p] = -1 - p;        // PTAG (high bit set)
    pi[(std::size_t)2 * stride + p] = p % 3;         // PSP
    pi[(std::size_t)3 * stride + p] = 0;             // PLEV
    pi[(std::size_t)4 * stride + p] = p % 2;         // PTAGH
  }
}

ParticleRestartState make_state() {
  ParticleRestartState s;
  s.next_tag_set = true; s.next_tag = 123456789012ull; s.tag_bound = 123456789999ull;
  s.rank = 0; s.gids = 0; s.nmb = 8;
  s.species_table = "nspecies = 3\nspecies.0 = tau_s 0.01\nspecies.1 = tau_s 0.1\n";
  s.resample[0] = 4; s.resample[1] = 17;
  s.x3_outflow_mass = 0.25; s.x3_outflow_count = 12; s.x3_removed[0] = 0.01; s.x3_removed[1] = 2;
  s.dropped_sum = {1e-3, -2e-3, 3e-3, 0.0};
  s.cloud_ord_status = 1; s.cloud_ord_sort_cycle = 40;
  s.cloud_ord = {2, 0, 1};
  s.cloud_ord_tag = {0x100000000ull, 7, 8};
  return s;
}

bool same_state(const ParticleRestartState &a, const ParticleRestartState &b) {
  return a.next_tag_set == b.next_tag_set && a.next_tag == b.next_tag && a.tag_bound == b.tag_bound &&
         a.rank == b.rank && a.gids == b.gids && a.nmb == b.nmb && a.merge_pass == b.merge_pass &&
         a.species_table == b.species_table && a.resample[0] == b.resample[0] &&
         a.resample[1] == b.resample[1] && a.x3_outflow_mass == b.x3_outflow_mass &&
         a.x3_outflow_count == b.x3_outflow_count && a.x3_removed[0] == b.x3_removed[0] &&
         a.x3_removed[1] == b.x3_removed[1] && a.dropped_sum == b.dropped_sum &&
         a.cloud_ord_status == b.cloud_ord_status &&
         a.cloud_ord_sort_cycle == b.cloud_ord_sort_cycle && a.cloud_ord == b.cloud_ord &&
         a.cloud_ord_tag == b.cloud_ord_tag &&
         std::memcmp(a.resample_clk_n, b.resample_clk_n, sizeof(a.resample_clk_n)) == 0 &&
         std::memcmp(a.merge_clk_n, b.merge_clk_n, sizeof(a.merge_clk_n)) == 0 &&
         std::memcmp(a.regrid_evt, b.regrid_evt, sizeof(a.regrid_evt)) == 0;
}

bool write_file(const std::string &path, const void *p, std::size_t n) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(p, 1, n, f) == n;
  return std::fclose(f) == 0 && ok;
}

// a version-1 section as the reference's earlier code wrote it: nidata 4 (no PTAGH), the int32
// record next_tag
std::vector<char> version1(int n, const std::vector<double> &pr, const std::vector<int> &pi,
                           long long stride) {
  std::vector<char> st, b;
  auto put = [](std::vector<char> &v, const void *p, std::size_t k) {
    const char *c = static_cast<const char *>(p);
    v.insert(v.end(), c, c + k);
  };
  char key[16] = {0};
  std::strncpy(key, "next_tag", 15);
  put(st, key, 16);
  const std::int32_t len = 4, tag = 4242;
  put(st, &len, 4);
  put(st, &tag, 4);
  put(b, "AKPRST01", 8);
  const std::int32_t head[6] = {1, 8, 4, 1, 17, 4};
  put(b, head, sizeof(head));
  const std::uint64_t total = 8 + 24 + 8 + 8 + 8 + 4 + st.size() + (std::uint64_t)n * (17 * 8 + 4 * 4) + 8;
  put(b, &total, 8);
  const std::int64_t np = n;
  put(b, &np, 8);
  const double dt = 0.5;
  put(b, &dt, 8);
  const std::int32_t ns = (std::int32_t)st.size();
  put(b, &ns, 4);
  put(b, st.data(), st.size());
  for (int r = 0; r < 17; ++r) put(b, pr.data() + (std::size_t)r * stride, (std::size_t)n * 8);
  for (int r = 0; r < 4; ++r) put(b, pi.data() + (std::size_t)r * stride, (std::size_t)n * 4);
  put(b, "AKPRST01", 8);
  return b;
}

int host_checks(const std::string &dir) {
  const int n = 1000;
  const long long stride = 1234;
  std::vector<double> pr;
  std::vector<int> pi;
  make_rows(n, stride, pr, pi);
  const ParticleRestartState st = make_state();
  std::vector<char> buf;
  std::string err = athenak_b200::PackParticleRestartRows(pr.data(), pi.data(), stride, n, 0.125, st, buf);
  check(err.empty(), "pack from host rows");
  ParticleRestartSection sec;
  err = athenak_b200::ParseParticleRestart(buf, sec);
  check(err.empty() && sec.version == 2 && sec.np == n && sec.dtnew == 0.125, "parse back");
  bool rows = true;
  for (int r = 0; r < 17; ++r)
    rows = rows && std::memcmp(&sec.pr[(std::size_t)r * n], &pr[(std::size_t)r * stride], n * 8) == 0;
  for (int r = 0; r < 5; ++r)
    rows = rows && std::memcmp(&sec.pi[(std::size_t)r * n], &pi[(std::size_t)r * stride], n * 4) == 0;
  check(rows, "rows bit for bit");
  check(same_state(st, sec.state) && sec.notes.empty(), "records");
  // the file and its rows for the reader of the test
  const long long hdr[2] = {n, stride};
  std::vector<char> rowfile((const char *)hdr, (const char *)hdr + sizeof(hdr));
  rowfile.insert(rowfile.end(), (const char *)pr.data(), (const char *)(pr.data() + pr.size()));
  rowfile.insert(rowfile.end(), (const char *)pi.data(), (const char *)(pi.data() + pi.size()));
  check(write_file(dir + "/host.rst", buf.data(), buf.size()) &&
        write_file(dir + "/host.rows", rowfile.data(), rowfile.size()), "files written");
  // version 1
  const std::vector<char> v1 = version1(n, pr, pi, stride);
  err = athenak_b200::ParseParticleRestart(v1, sec);
  bool v1ok = err.empty() && sec.version == 1 && sec.nidata == 4 && sec.state.next_tag_set &&
              sec.state.next_tag == 4242 && sec.dtnew == 0.5;
  for (int p = 0; p < n && v1ok; ++p)
    v1ok = sec.pi[(std::size_t)4 * n + p] == 0 && sec.pi[(std::size_t)1 * n + p] == pi[(std::size_t)stride + p];
  check(v1ok, "version-1 section (no high tag words, int32 counter)");
  // damaged sections
  std::vector<char> cut(buf.begin(), buf.end() - 9);
  cut.insert(cut.end(), buf.end() - 8, buf.end());
  check(!athenak_b200::ParseParticleRestart(cut, sec).empty(), "truncated section rejected");
  std::vector<char> magic = buf;
  magic[0] = 'X';
  check(!athenak_b200::ParseParticleRestart(magic, sec).empty(), "bad magic rejected");
  std::vector<char> cols = buf;
  const std::int32_t nr = 16;
  std::memcpy(cols.data() + 8 + 4 * 4, &nr, 4);
  check(!athenak_b200::ParseParticleRestart(cols, sec).empty(), "other column count rejected");
  std::vector<char> rec = buf;   // the size of rank_blocks (the second record) changed
  const std::size_t at2 = 8 + 24 + 8 + 8 + 8 + 4 + (16 + 4 + 24) + 16;
  const std::int32_t wrong = 8;
  std::memcpy(rec.data() + at2, &wrong, 4);
  check(!athenak_b200::ParseParticleRestart(rec, sec).empty(), "record of a wrong size rejected");
  return bad;
}

int device_checks() {
  const int n = 5000;
  const long long stride = n + 77, stride2 = n + 1000;
  std::vector<double> pr;
  std::vector<int> pi;
  make_rows(n, stride, pr, pi);
  double *d_pr = nullptr, *d_pr2 = nullptr;
  int *d_pi = nullptr, *d_pi2 = nullptr;
  if (cudaMalloc(&d_pr, pr.size() * 8) != cudaSuccess || cudaMalloc(&d_pi, pi.size() * 4) != cudaSuccess ||
      cudaMalloc(&d_pr2, (std::size_t)17 * stride2 * 8) != cudaSuccess ||
      cudaMalloc(&d_pi2, (std::size_t)5 * stride2 * 4) != cudaSuccess) {
    check(false, "device allocation");
    return bad;
  }
  cudaMemcpy(d_pr, pr.data(), pr.size() * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(d_pi, pi.data(), pi.size() * 4, cudaMemcpyHostToDevice);
  dustb_ctx c;
  std::memset(&c, 0, sizeof(c));
  c.part.pr = d_pr; c.part.pi = d_pi; c.part.stride = stride; c.part.npart = n;
  std::vector<char> buf;
  std::string err = athenak_b200::PackParticleRestart(c, nullptr, 0.25, make_state(), buf);
  check(err.empty(), "pack from the device");
  ParticleRestartSection sec;
  err = athenak_b200::ParseParticleRestart(buf, sec);
  dustb_ctx c2 = c;
  c2.part.pr = d_pr2; c2.part.pi = d_pi2; c2.part.stride = stride2; c2.part.npart = 0;
  if (err.empty()) err = athenak_b200::RestoreParticleRows(sec, c2, nullptr);
  check(err.empty() && c2.part.npart == n, "restore into arrays of another capacity");
  std::vector<double> back((std::size_t)17 * stride2);
  std::vector<int> iback((std::size_t)5 * stride2);
  cudaMemcpy(back.data(), d_pr2, back.size() * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(iback.data(), d_pi2, iback.size() * 4, cudaMemcpyDeviceToHost);
  bool same = true;
  for (int r = 0; r < 17; ++r)
    same = same && std::memcmp(&back[(std::size_t)r * stride2], &pr[(std::size_t)r * stride], n * 8) == 0;
  for (int r = 0; r < 5; ++r)
    same = same && std::memcmp(&iback[(std::size_t)r * stride2], &pi[(std::size_t)r * stride], n * 4) == 0;
  check(same, "device rows bit for bit after the round trip");
  dustb_ctx small = c2;
  small.part.stride = n - 1;
  check(!athenak_b200::RestoreParticleRows(sec, small, nullptr).empty(), "too small arrays rejected");
  cudaFree(d_pr); cudaFree(d_pi); cudaFree(d_pr2); cudaFree(d_pi2);
  return bad;
}

// the rows of one writing rank: n particles of blocks [gids, gids + nmb), tags from tag0
void rank_rows(int n, int gids, int nmb, int tag0, std::vector<double> &pr, std::vector<int> &pi) {
  make_rows(n, n, pr, pi);
  for (int p = 0; p < n; ++p) {
    pi[p] = gids + (p * 7) % nmb;
    pi[(std::size_t)1 * n + p] = tag0 + p;
    pr[p] += 100.0 * gids;                   // rows told apart by rank
  }
}

// one particle of a parsed section (rows r * np + p) against one of the writer's rows
bool same_particle(const ParticleRestartSection &s, std::int64_t p, const std::vector<double> &pr,
                   const std::vector<int> &pi, int n, int q) {
  bool ok = true;
  for (int r = 0; r < 17; ++r) ok = ok && s.pr[(std::size_t)r * s.np + p] == pr[(std::size_t)r * n + q];
  for (int r = 0; r < 5; ++r) ok = ok && s.pi[(std::size_t)r * s.np + p] == pi[(std::size_t)r * n + q];
  return ok;
}

// a file of two sections (ranks 0 and 1 of a run on two ranks, blocks [0, 4) and [4, 8)) after
// other bytes; read back on two ranks with the same blocks (each its own section exactly), on
// one rank (every particle, the records of section 0, a new tag counter, no cloud order), on
// two ranks with other blocks (the particles of each rank's blocks from both sections, in
// section order); damaged files and a rank count that does not match rejected
int rank_checks(const std::string &dir) {
  const int n0 = 10, n1 = 7;
  std::vector<double> pr0, pr1;
  std::vector<int> pi0, pi1;
  rank_rows(n0, 0, 4, 1000, pr0, pi0);
  rank_rows(n1, 4, 4, 2000, pr1, pi1);
  ParticleRestartState s0 = make_state(), s1 = make_state();
  s0.nranks = s1.nranks = 2;
  s0.rank = 0; s0.gids = 0; s0.nmb = 4; s0.next_tag = 1010; s0.merge_pass = 3;
  s1.rank = 1; s1.gids = 4; s1.nmb = 4; s1.next_tag = 2007; s1.merge_pass = 5;
  std::vector<char> b0, b1, file(100, 'm');   // (the mesh data before the sections)
  std::string err = athenak_b200::PackParticleRestartRows(pr0.data(), pi0.data(), n0, n0, 0.25, s0, b0);
  err += athenak_b200::PackParticleRestartRows(pr1.data(), pi1.data(), n1, n1, 0.5, s1, b1);
  check(err.empty(), "two ranks' sections packed");
  file.insert(file.end(), b0.begin(), b0.end());
  file.insert(file.end(), b1.begin(), b1.end());
  std::vector<std::vector<char>> secs;
  err = athenak_b200::SplitParticleRestart(file, 100, secs);
  check(err.empty() && secs.size() == 2 && secs[0] == b0 && secs[1] == b1, "file split into its sections");
  ParticleRestartSection one;
  check(!athenak_b200::ParseParticleRestart(secs[0], one).empty() &&
        athenak_b200::ParseParticleRestart(secs[0], one, 2).empty() && one.state.nranks == 2,
        "a section's rank count is checked");
  // two ranks, the writer's blocks: exact
  bool m0 = false, m1 = false;
  err = athenak_b200::ParticleRestartOwnSectionMatches(secs, 0, 2, 0, 4, m0);
  err += athenak_b200::ParticleRestartOwnSectionMatches(secs, 1, 2, 4, 4, m1);
  check(err.empty() && m0 && m1, "own sections match on the writer's layout");
  ParticleRestartSection e0, e1;
  err = athenak_b200::SelectParticleRestart(secs, 0, 0, 4, true, e0);
  err += athenak_b200::SelectParticleRestart(secs, 1, 4, 4, true, e1);
  bool ok = err.empty() && e0.np == n0 && e1.np == n1 && e0.dtnew == 0.25 && e1.dtnew == 0.5 &&
            e0.state.next_tag == 1010 && e1.state.next_tag == 2007 && e1.state.merge_pass == 5 &&
            e1.state.cloud_ord == s1.cloud_ord;
  for (int p = 0; p < n0 && ok; ++p) ok = same_particle(e0, p, pr0, pi0, n0, p);
  for (int p = 0; p < n1 && ok; ++p) ok = same_particle(e1, p, pr1, pi1, n1, p);
  check(ok, "exact: each rank its own section, rows and records bit for bit");
  // one rank: no match (two sections), everything gathered
  bool m = true;
  err = athenak_b200::ParticleRestartOwnSectionMatches(secs, 0, 1, 0, 8, m);
  ParticleRestartSection all;
  err += athenak_b200::SelectParticleRestart(secs, 0, 0, 8, m, all);
  ok = err.empty() && !m && all.np == n0 + n1 && all.dtnew == 0.25 && all.state.merge_pass == 3 &&
       !all.state.next_tag_set && all.state.next_tag == 0 && all.state.cloud_ord.empty() &&
       all.state.cloud_ord_tag.empty() && all.state.cloud_ord_status == 0;
  for (int p = 0; p < n0 && ok; ++p) ok = same_particle(all, p, pr0, pi0, n0, p);
  for (int p = 0; p < n1 && ok; ++p) ok = same_particle(all, n0 + p, pr1, pi1, n1, p);
  check(ok, "one rank: every particle in section order, section 0's records, tag counter anew");
  // two ranks, blocks [0, 3) and [3, 8): no match, each rank its blocks from both sections
  err = athenak_b200::ParticleRestartOwnSectionMatches(secs, 0, 2, 0, 3, m0);
  err += athenak_b200::ParticleRestartOwnSectionMatches(secs, 1, 2, 3, 5, m1);
  ParticleRestartSection g0, g1;
  err += athenak_b200::SelectParticleRestart(secs, 0, 0, 3, m0 && m1, g0);
  err += athenak_b200::SelectParticleRestart(secs, 1, 3, 5, m0 && m1, g1);
  std::vector<std::pair<int, int>> want0, want1;   // (section, particle)
  for (int p = 0; p < n0; ++p) (pi0[p] < 3 ? want0 : want1).emplace_back(0, p);
  for (int p = 0; p < n1; ++p) (pi1[p] < 3 ? want0 : want1).emplace_back(1, p);
  ok = err.empty() && !m0 && !m1 && g0.np == (std::int64_t)want0.size() &&
       g1.np == (std::int64_t)want1.size() && g1.state.merge_pass == 3 && !g1.state.next_tag_set;
  for (std::size_t q = 0; q < want0.size() && ok; ++q)
    ok = want0[q].first == 0 ? same_particle(g0, q, pr0, pi0, n0, want0[q].second)
                             : same_particle(g0, q, pr1, pi1, n1, want0[q].second);
  for (std::size_t q = 0; q < want1.size() && ok; ++q)
    ok = want1[q].first == 0 ? same_particle(g1, q, pr0, pi0, n0, want1[q].second)
                             : same_particle(g1, q, pr1, pi1, n1, want1[q].second);
  check(ok && !want0.empty() && !want1.empty(), "other blocks: each rank's particles from both sections");
  // a particle outside the blocks on the exact path, a truncated file, a section too many
  std::vector<char> bad0;
  pi0[3] = 6;
  athenak_b200::PackParticleRestartRows(pr0.data(), pi0.data(), n0, n0, 0.25, s0, bad0);
  std::vector<std::vector<char>> badsecs = {bad0, b1};
  ParticleRestartSection x;
  check(!athenak_b200::SelectParticleRestart(badsecs, 0, 0, 4, true, x).empty(),
        "exact: a particle of another block rejected");
  std::vector<char> cut(file.begin(), file.end() - 9);
  std::vector<std::vector<char>> cs;
  check(!athenak_b200::SplitParticleRestart(cut, 100, cs).empty(), "truncated file rejected");
  std::vector<std::vector<char>> three = {b0, b1, b1};
  ParticleRestartSection y;
  check(!athenak_b200::SelectParticleRestart(three, 0, 0, 8, false, y).empty(),
        "sections whose rank count is not their number rejected");
  return write_file(dir + "/ranks.rst", file.data() + 100, file.size() - 100) ? bad : bad + 1;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::printf("usage: restart_tool host|ranks|device <dir>\n");
    return 2;
  }
  const std::string mode = argv[1];
  const int b = (mode == "host") ? host_checks(argv[2])
              : (mode == "ranks") ? rank_checks(argv[2]) : device_checks();
  return b ? 1 : 0;
}
