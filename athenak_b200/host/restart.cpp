// restart.cpp -- the particle section of the restart file; see restart.hpp.
#include "restart.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <functional>
#include <map>
#include <type_traits>

namespace athenak_b200 {
namespace {

const char kMagic[9] = "AKPRST01";
constexpr std::int32_t kVersion = 2;
constexpr std::size_t kHeadBytes = 8 + 6 * sizeof(std::int32_t) + sizeof(std::uint64_t);
constexpr std::size_t kStateMax = 0x7fffffff;   // the dust state's length is an int32
constexpr int kNReal = 17, kNInt = 5;

// appends raw bytes to a section under construction
void Put(std::vector<char> &b, const void *p, std::size_t n) {
  const char *c = static_cast<const char *>(p);
  b.insert(b.end(), c, c + n);
}
template <typename T>
void PutValue(std::vector<char> &b, const T &v) { Put(b, &v, sizeof(T)); }

// one framed record: the name NUL-padded to 16 bytes, the payload length as int32, the payload
void PutRecord(std::vector<char> &b, const char *name, const void *payload, std::size_t n) {
  std::string frame(16, '\0');
  frame.replace(0, std::min<std::size_t>(15, std::strlen(name)), name,
                std::min<std::size_t>(15, std::strlen(name)));
  const std::int32_t len = static_cast<std::int32_t>(n);
  b.reserve(b.size() + frame.size() + sizeof(len) + n);
  Put(b, frame.data(), frame.size());
  Put(b, &len, sizeof(len));
  Put(b, payload, n);
}

// the dust records in the reference's order (PackRestartState, then the cell-order index)
void PackState(const ParticleRestartState &s, std::vector<char> &b) {
  const std::uint64_t ts[3] = {s.next_tag_set ? 1ULL : 0ULL, s.next_tag, s.tag_bound};
  PutRecord(b, "tag_state", ts, sizeof(ts));
  const std::int32_t rb[3] = {s.rank, s.gids, s.nmb};
  PutRecord(b, "rank_blocks", rb, sizeof(rb));
  PutRecord(b, "merge_pass", &s.merge_pass, sizeof(s.merge_pass));
  PutRecord(b, "species_table", s.species_table.data(), s.species_table.size());
  if (!s.mroot.empty()) PutRecord(b, "mroot", s.mroot.data(), s.mroot.size() * sizeof(double));
  if (!s.imex_mown.empty())
    PutRecord(b, "imex_mown", s.imex_mown.data(), s.imex_mown.size() * sizeof(double));
  PutRecord(b, "resample", s.resample, sizeof(s.resample));
  char clk[sizeof(s.resample_clk_r) + sizeof(s.resample_clk_n)];
  std::memcpy(clk, s.resample_clk_r, sizeof(s.resample_clk_r));
  std::memcpy(clk + sizeof(s.resample_clk_r), s.resample_clk_n, sizeof(s.resample_clk_n));
  PutRecord(b, "resample_clk", clk, sizeof(clk));
  char mclk[sizeof(s.merge_clk_r) + sizeof(s.merge_clk_n)];
  std::memcpy(mclk, s.merge_clk_r, sizeof(s.merge_clk_r));
  std::memcpy(mclk + sizeof(s.merge_clk_r), s.merge_clk_n, sizeof(s.merge_clk_n));
  PutRecord(b, "merge_clk", mclk, sizeof(mclk));
  if (!s.amr_state.empty())
    PutRecord(b, "amr_state", s.amr_state.data(), s.amr_state.size() * sizeof(std::int32_t));
  PutRecord(b, "split", s.split, sizeof(s.split));
  PutRecord(b, "coarsen_n", s.coarsen, sizeof(s.coarsen));
  PutRecord(b, "amr_regrids", &s.amr_regrids, sizeof(s.amr_regrids));
  PutRecord(b, "regrid_evt", s.regrid_evt, sizeof(s.regrid_evt));
  PutRecord(b, "regrid_evt_t", s.regrid_evt_t, sizeof(s.regrid_evt_t));
  std::vector<double> led(5 + s.dropped_sum.size());
  led[0] = s.x3_outflow_mass; led[1] = s.x3_outflow_count;
  led[2] = s.x3_removed[0]; led[3] = s.x3_removed[1];
  led[4] = static_cast<double>(s.dropped_sum.size());
  for (std::size_t v = 0; v < s.dropped_sum.size(); ++v) led[5 + v] = s.dropped_sum[v];
  PutRecord(b, "x3_ledger", led.data(), led.size() * sizeof(double));
  if (s.cloud_ord_status != 0) {
    const bool stored = s.cloud_ord_status == 1;
    const std::int32_t info[3] = {s.cloud_ord_status,
                                  stored ? static_cast<std::int32_t>(s.cloud_ord.size()) : 0,
                                  s.cloud_ord_sort_cycle};
    PutRecord(b, "cloud_ord_n", info, sizeof(info));
    if (stored) {
      PutRecord(b, "cloud_ord", s.cloud_ord.data(), s.cloud_ord.size() * sizeof(std::int32_t));
      PutRecord(b, "cloud_ord_tag", s.cloud_ord_tag.data(),
                s.cloud_ord_tag.size() * sizeof(std::uint64_t));
    }
  }
}

// The dust records of a section: frames of a 16-byte name, an int32 length and the payload.
// Each known name has a decoder that checks the payload's size and stores it in the state;
// an unknown name is kept as read.  "" or the error.
std::string UnpackState(const char *p, std::size_t nbytes, ParticleRestartSection &sec) {
  ParticleRestartState &s = sec.state;
  using Decoder = std::function<bool(const char *, std::size_t)>;
  // a payload of exactly `want` bytes copied into dst
  auto exact = [](void *dst, std::size_t want) -> Decoder {
    return [dst, want](const char *d, std::size_t n) {
      if (n != want) return false;
      std::memcpy(dst, d, want);
      return true;
    };
  };
  // a payload of whole items of type T into a vector
  auto items = [](auto &vec) -> Decoder {
    return [&vec](const char *d, std::size_t n) {
      using T = typename std::decay_t<decltype(vec)>::value_type;
      if (n % sizeof(T) != 0) return false;
      vec.resize(n / sizeof(T));
      if (n) std::memcpy(vec.data(), d, n);
      return true;
    };
  };
  // two fixed arrays stored back to back
  auto pair = [](void *a, std::size_t na, void *b, std::size_t nb) -> Decoder {
    return [=](const char *d, std::size_t n) {
      if (n != na + nb) return false;
      std::memcpy(a, d, na);
      std::memcpy(b, d + na, nb);
      return true;
    };
  };
  bool species_found = false;
  std::int32_t rank_blocks[3] = {0, 0, 0}, cloud_info[3] = {0, 0, 0};
  std::uint64_t tag_state[3] = {0, 0, 0};
  const std::map<std::string, Decoder> decoders = {
      {"next_tag", [&](const char *d, std::size_t n) {   // version 1: int32, -1 when unset
         std::int32_t v = 0;
         if (!exact(&v, sizeof(v))(d, n)) return false;
         s.next_tag_set = v >= 0;
         s.next_tag = v >= 0 ? static_cast<std::uint64_t>(v) : 0;
         return true;
       }},
      {"tag_state", [&](const char *d, std::size_t n) {
         if (!exact(tag_state, sizeof(tag_state))(d, n)) return false;
         s.next_tag_set = tag_state[0] != 0;
         s.next_tag = tag_state[1];
         s.tag_bound = tag_state[2];
         return true;
       }},
      {"rank_blocks", [&](const char *d, std::size_t n) {
         s.rank_blocks_read = exact(rank_blocks, sizeof(rank_blocks))(d, n);
         s.rank = rank_blocks[0]; s.gids = rank_blocks[1]; s.nmb = rank_blocks[2];
         return s.rank_blocks_read;
       }},
      {"merge_pass", exact(&s.merge_pass, sizeof(s.merge_pass))},
      {"species_table", [&](const char *d, std::size_t n) {
         species_found = true;
         s.species_table.assign(d, n);
         return true;
       }},
      {"mroot", items(s.mroot)},
      {"imex_mown", items(s.imex_mown)},
      {"resample", exact(s.resample, sizeof(s.resample))},
      {"resample_clk", pair(s.resample_clk_r, sizeof(s.resample_clk_r), s.resample_clk_n,
                            sizeof(s.resample_clk_n))},
      {"merge_clk", pair(s.merge_clk_r, sizeof(s.merge_clk_r), s.merge_clk_n,
                         sizeof(s.merge_clk_n))},
      {"amr_state", [&](const char *d, std::size_t n) {
         // [flag, count, count values]
         if (n < 2 * sizeof(std::int32_t) || !items(s.amr_state)(d, n)) return false;
         return static_cast<std::size_t>(s.amr_state[1]) + 2 == s.amr_state.size();
       }},
      {"split", exact(s.split, sizeof(s.split))},
      {"coarsen_n", exact(s.coarsen, sizeof(s.coarsen))},
      {"amr_regrids", exact(&s.amr_regrids, sizeof(s.amr_regrids))},
      {"regrid_evt", exact(s.regrid_evt, sizeof(s.regrid_evt))},
      {"regrid_evt_t", exact(s.regrid_evt_t, sizeof(s.regrid_evt_t))},
      {"x3_ledger", [&](const char *d, std::size_t n) {
         // outflow mass and count, the removed (mass, count), the number of dropped sums,
         // then those sums
         std::vector<double> led;
         if (n < 5 * sizeof(double) || !items(led)(d, n)) return false;
         const int ndrop = static_cast<int>(led[4]);
         if (ndrop < 0 || static_cast<std::size_t>(5 + ndrop) != led.size()) return false;
         s.x3_outflow_mass = led[0]; s.x3_outflow_count = led[1];
         s.x3_removed[0] = led[2]; s.x3_removed[1] = led[3];
         s.dropped_sum.assign(led.begin() + 5, led.end());
         return true;
       }},
      {"cloud_ord_n", [&](const char *d, std::size_t n) {
         if (!exact(cloud_info, sizeof(cloud_info))(d, n)) return false;
         s.cloud_ord_status = cloud_info[0];
         s.cloud_ord_sort_cycle = cloud_info[2];
         return true;
       }},
      {"cloud_ord", items(s.cloud_ord)},
      {"cloud_ord_tag", items(s.cloud_ord_tag)},
  };
  constexpr std::size_t kFrame = 16 + sizeof(std::int32_t);
  std::size_t at = 0;
  while (at + kFrame <= nbytes) {
    char raw_name[17] = {0};
    std::memcpy(raw_name, p + at, 16);
    std::int32_t len = 0;
    std::memcpy(&len, p + at + 16, sizeof(len));
    if (len < 0 || at + kFrame + static_cast<std::size_t>(len) > nbytes)
      return "dust record runs past the end";
    const std::string name(raw_name);
    const char *payload = p + at + kFrame;
    const std::size_t n = static_cast<std::size_t>(len);
    const auto it = decoders.find(name);
    if (it == decoders.end()) {
      s.other.emplace_back(name, std::vector<char>(payload, payload + n));
      sec.notes.push_back("record '" + name + "' is not known to this code and is kept as read");
    } else if (!it->second(payload, n)) {
      return "dust record " + name + " has an unexpected size";
    }
    at += kFrame + n;
  }
  if (!species_found) sec.notes.push_back("no record species_table (an older file)");
  // the index must be a whole group: stored with both arrays of its length
  if (s.cloud_ord_status == 1 &&
      (s.cloud_ord.size() != s.cloud_ord_tag.size() || s.cloud_ord.empty())) {
    sec.notes.push_back("cloud order records are incomplete: the index is rebuilt");
    s.cloud_ord_status = 0;
    s.cloud_ord.clear();
    s.cloud_ord_tag.clear();
  }
  return "";
}

}  // namespace

std::string PackParticleRestartRows(const double *pr, const int *pi, long long stride,
                                    std::int64_t np, double dtnew,
                                    const ParticleRestartState &st, std::vector<char> &buf) {
  if (np < 0 || stride < np || (np > 0 && (!pr || !pi))) return "restart: bad particle rows";
  if (st.nranks < 1 || st.rank < 0 || st.rank >= st.nranks)
    return "restart: the writing rank or the rank count is out of range";
  std::vector<char> state;
  PackState(st, state);
  if (state.size() > kStateMax) return "restart: the dust records exceed the int32 length";
  buf.clear();
  const std::uint64_t rows = static_cast<std::uint64_t>(np) * (kNReal * sizeof(double) +
                                                               kNInt * sizeof(int));
  const std::uint64_t total = kHeadBytes + sizeof(std::int64_t) + sizeof(double) +
                              sizeof(std::int32_t) + state.size() + rows + 8;
  buf.reserve(total);
  Put(buf, kMagic, 8);
  const std::int32_t head[6] = {kVersion, static_cast<std::int32_t>(sizeof(double)),
                                static_cast<std::int32_t>(sizeof(int)), st.nranks, kNReal, kNInt};
  Put(buf, head, sizeof(head));
  PutValue(buf, total);
  PutValue(buf, np);
  PutValue(buf, dtnew);
  PutValue(buf, static_cast<std::int32_t>(state.size()));
  Put(buf, state.data(), state.size());
  for (int c = 0; c < kNReal; ++c) Put(buf, pr + (std::size_t)c * stride, (std::size_t)np * sizeof(double));
  for (int c = 0; c < kNInt; ++c) Put(buf, pi + (std::size_t)c * stride, (std::size_t)np * sizeof(int));
  Put(buf, kMagic, 8);
  if (buf.size() != total) return "restart: internal size mismatch";
  return "";
}

std::string PackParticleRestart(const dustb_ctx &ctx, void *stream, double dtnew,
                                const ParticleRestartState &st, std::vector<char> &buf) {
  const std::int64_t np = ctx.part.npart;
  std::vector<double> pr((std::size_t)np * kNReal);
  std::vector<int> pi((std::size_t)np * kNInt);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int c = 0; c < kNReal && np > 0; ++c)
    if (cudaMemcpyAsync(pr.data() + (std::size_t)c * np, ctx.part.pr + (std::size_t)c * ctx.part.stride,
                        (std::size_t)np * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return "restart: particle rows not copied";
  for (int c = 0; c < kNInt && np > 0; ++c)
    if (cudaMemcpyAsync(pi.data() + (std::size_t)c * np, ctx.part.pi + (std::size_t)c * ctx.part.stride,
                        (std::size_t)np * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return "restart: particle rows not copied";
  if (cudaStreamSynchronize(s) != cudaSuccess) return "restart: particle rows not copied";
  return PackParticleRestartRows(pr.data(), pi.data(), np, np, dtnew, st, buf);
}

std::string ParseParticleRestart(const std::vector<char> &buf, ParticleRestartSection &out,
                                 int nsec) {
  out = ParticleRestartSection();
  if (nsec < 1) return "restart: no particle section";
  if (buf.size() < kHeadBytes + 8 || std::memcmp(buf.data(), kMagic, 8) != 0 ||
      std::memcmp(buf.data() + buf.size() - 8, kMagic, 8) != 0)
    return "restart: missing or truncated particle section (no head or end marker)";
  std::int32_t head[6];
  std::memcpy(head, buf.data() + 8, sizeof(head));
  std::uint64_t total = 0;
  std::memcpy(&total, buf.data() + 8 + sizeof(head), sizeof(total));
  const bool columns_ok = head[5] == kNInt || (head[0] == 1 && head[5] == kNInt - 1);
  if ((head[0] != 1 && head[0] != 2) || head[1] != (std::int32_t)sizeof(double) ||
      head[2] != (std::int32_t)sizeof(int) || head[3] != nsec || head[4] != kNReal || !columns_ok)
    return "restart: version, type sizes, rank count or particle columns do not match (file: "
           "version " + std::to_string(head[0]) + ", Real " + std::to_string(head[1]) +
           " bytes, int " + std::to_string(head[2]) + " bytes, ranks " + std::to_string(head[3]) +
           ", nrdata " + std::to_string(head[4]) + ", nidata " + std::to_string(head[5]) + ")";
  out.version = head[0]; out.ranks = head[3]; out.nrdata = head[4]; out.nidata = head[5];
  std::size_t at = kHeadBytes;
  std::int32_t nstate = 0;
  std::memcpy(&out.np, buf.data() + at, sizeof(out.np)); at += sizeof(out.np);
  std::memcpy(&out.dtnew, buf.data() + at, sizeof(out.dtnew)); at += sizeof(out.dtnew);
  std::memcpy(&nstate, buf.data() + at, sizeof(nstate)); at += sizeof(nstate);
  if (out.np < 0 || nstate < 0) return "restart: sizes inside the section are inconsistent";
  const std::size_t need = at + (std::size_t)nstate +
                           (std::size_t)out.np * (kNReal * sizeof(double) + out.nidata * sizeof(int)) + 8;
  if (need != buf.size() || total != buf.size())
    return "restart: sizes inside the section are inconsistent";
  std::string err = UnpackState(buf.data() + at, (std::size_t)nstate, out);
  if (!err.empty()) return "restart: " + err;
  out.state.nranks = head[3];
  at += (std::size_t)nstate;
  const std::size_t n = (std::size_t)out.np;
  out.pr.resize(n * kNReal);
  if (n) std::memcpy(out.pr.data(), buf.data() + at, n * kNReal * sizeof(double));
  at += n * kNReal * sizeof(double);
  out.pi.assign(n * kNInt, 0);   // version 1: PTAGH (the last row) stays 0
  if (n) std::memcpy(out.pi.data(), buf.data() + at, n * out.nidata * sizeof(int));
  return "";
}

std::string RestoreParticleRows(const ParticleRestartSection &sec, dustb_ctx &ctx, void *stream) {
  const std::int64_t np = sec.np;
  if (np > ctx.part.stride) return "restart: the particle arrays cannot hold the section's rows";
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int c = 0; c < kNReal && np > 0; ++c)
    if (cudaMemcpyAsync(ctx.part.pr + (std::size_t)c * ctx.part.stride, sec.pr.data() + (std::size_t)c * np,
                        (std::size_t)np * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return "restart: particle rows not restored";
  for (int c = 0; c < kNInt && np > 0; ++c)
    if (cudaMemcpyAsync(ctx.part.pi + (std::size_t)c * ctx.part.stride, sec.pi.data() + (std::size_t)c * np,
                        (std::size_t)np * sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess)
      return "restart: particle rows not restored";
  if (cudaStreamSynchronize(s) != cudaSuccess) return "restart: particle rows not restored";
  ctx.part.npart = static_cast<int>(np);
  return "";
}

std::string SplitParticleRestart(const std::vector<char> &file, std::size_t at,
                                 std::vector<std::vector<char>> &sections) {
  sections.clear();
  while (at < file.size()) {
    if (file.size() - at < kHeadBytes + 8 || std::memcmp(file.data() + at, kMagic, 8) != 0)
      return "restart: particle section " + std::to_string(sections.size()) +
             " has no head at byte " + std::to_string(at);
    std::uint64_t total = 0;
    std::memcpy(&total, file.data() + at + 8 + 6 * sizeof(std::int32_t), sizeof(total));
    if (total < kHeadBytes + 8 || total > file.size() - at)
      return "restart: particle section " + std::to_string(sections.size()) +
             " runs past the end of the file";
    sections.emplace_back(file.begin() + (std::ptrdiff_t)at,
                          file.begin() + (std::ptrdiff_t)(at + total));
    at += total;
  }
  if (sections.empty()) return "restart: no particle section";
  return "";
}

std::string ParticleRestartOwnSectionMatches(const std::vector<std::vector<char>> &sections,
                                             int me, int nranks, int gids, int nmb,
                                             bool &match) {
  match = false;
  const int nsec = static_cast<int>(sections.size());
  if (nsec < 1) return "restart: no particle section";
  if (nranks < 1 || me < 0 || me >= nranks || nmb < 0) return "restart: bad rank or blocks";
  if (nsec != nranks) return "";
  ParticleRestartSection own;
  std::string err = ParseParticleRestart(sections[me], own, nsec);
  if (!err.empty()) return err;
  // one rank: also sections written before the rank_blocks record existed
  match = nranks == 1 || (own.state.rank_blocks_read && own.state.rank == me &&
                          own.state.gids == gids && own.state.nmb == nmb);
  return "";
}

std::string SelectParticleRestart(const std::vector<std::vector<char>> &sections, int me,
                                  int gids, int nmb, bool exact, ParticleRestartSection &out) {
  out = ParticleRestartSection();
  const int nsec = static_cast<int>(sections.size());
  if (nsec < 1) return "restart: no particle section";
  if (me < 0 || nmb < 0 || (exact && me >= nsec)) return "restart: bad rank or blocks";
  auto mine = [&](int gid) { return gid >= gids && gid < gids + nmb; };
  if (exact) {
    std::string err = ParseParticleRestart(sections[me], out, nsec);
    if (!err.empty()) return err;
    for (std::int64_t p = 0; p < out.np; ++p)
      if (!mine(out.pi[(std::size_t)p]))
        return "restart: a particle names a MeshBlock that does not exist (particle " +
               std::to_string(p) + ", block " + std::to_string(out.pi[(std::size_t)p]) + ")";
    return "";
  }
  // the rows kept, row by row, then packed into the section's layout (row r at r * np)
  std::vector<std::vector<double>> rc(kNReal);
  std::vector<std::vector<int>> ic(kNInt);
  for (int k = 0; k < nsec; ++k) {
    ParticleRestartSection s;
    std::string err = ParseParticleRestart(sections[k], s, nsec);
    if (!err.empty()) return "restart: section " + std::to_string(k) + ": " + err;
    if (k == 0) {
      out.version = s.version; out.ranks = s.ranks; out.nrdata = s.nrdata;
      out.nidata = s.nidata; out.dtnew = s.dtnew;
      out.state = s.state;
      out.notes = s.notes;
    }
    const std::size_t n = (std::size_t)s.np;
    for (std::size_t p = 0; p < n; ++p) {
      if (!mine(s.pi[p])) continue;   // PGID is row 0 of the integers
      for (int c = 0; c < kNReal; ++c) rc[c].push_back(s.pr[(std::size_t)c * n + p]);
      for (int c = 0; c < kNInt; ++c) ic[c].push_back(s.pi[(std::size_t)c * n + p]);
    }
  }
  const std::size_t np = rc[0].size();
  out.np = static_cast<std::int64_t>(np);
  out.pr.resize(np * kNReal);
  out.pi.resize(np * kNInt);
  for (int c = 0; c < kNReal; ++c)
    std::copy(rc[c].begin(), rc[c].end(), out.pr.begin() + (std::ptrdiff_t)(c * np));
  for (int c = 0; c < kNInt; ++c)
    std::copy(ic[c].begin(), ic[c].end(), out.pi.begin() + (std::ptrdiff_t)(c * np));
  // the sections' tag counters were per rank: the counter starts again; the cell-order index
  // of another layout is rebuilt
  out.state.next_tag_set = false;
  out.state.next_tag = 0;
  out.state.cloud_ord_status = 0;
  out.state.cloud_ord.clear();
  out.state.cloud_ord_tag.clear();
  return "";
}

}  // namespace athenak_b200
