// restart.hpp -- the particle section of the restart file ("AKPRST01", version 2), as the
// reference's dust module appends it after the MeshBlock data (src/dust/dust_restart.cpp):
//
//   char[8] "AKPRST01"; int32 version, sizeof(Real), sizeof(int), ranks written, nrdata, nidata
//   uint64 bytes of the whole section; int64 particles; Real particle time step (dtnew)
//   int32 bytes of the dust state, then the records (char[16] name, int32 bytes, data)
//   Real rows (nrdata rows of N), int rows (nidata rows of N); char[8] "AKPRST01"
//
// One rank writes one section.  Every real and integer row is written, so the particles come
// back bit for bit.  The dust records are those the reference writes, in its order; the ones
// that describe refinable clouds, resampling and mesh refinement (not part of this build) are
// written with the values of a run that has none of them and kept as they were read.  The
// cell-order index of the cloud kernels (cloud_ord_n / cloud_ord / cloud_ord_tag) is written
// when given.  Version 1 sections (int32 tags, nidata 4, record next_tag) are read too.
#ifndef ATHENAK_B200_RESTART_HPP_
#define ATHENAK_B200_RESTART_HPP_

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dustb.h"

namespace athenak_b200 {

struct ParticleRestartState {
  // tag_state: {counter set, next tag of this rank, bound above every tag issued}
  bool next_tag_set = false;
  std::uint64_t next_tag = 0, tag_bound = 0;
  // rank_blocks: {rank, first gid, blocks} (rank_blocks_read: the record was in the section)
  std::int32_t rank = 0, gids = 0, nmb = 0;
  bool rank_blocks_read = false;
  // the head's "ranks written": the number of sections of the file, one per writing rank
  std::int32_t nranks = 1;
  std::int32_t merge_pass = 0;
  std::string species_table;              // the resolved species table, ASCII lines
  std::vector<double> mroot, imex_mown;   // written when not empty
  std::uint64_t resample[2] = {0, 0};     // passes, particles removed
  double resample_clk_r[2] = {0.0, 0.0};  // origin, interval
  std::int64_t resample_clk_n[4] = {0, -1, 0, 0};   // by time, next, events, skipped
  double merge_clk_r[3] = {0.0, 0.0, 0.0};          // origin, interval, burst until
  std::int64_t merge_clk_n[2] = {0, -1};            // by time, next
  std::vector<std::int32_t> amr_state;    // written when not empty (adaptive meshes)
  std::uint64_t split[4] = {0, 0, 0, 0};
  std::uint64_t coarsen[4] = {0, 0, 0, 0};
  std::int32_t amr_regrids = 0;
  std::int64_t regrid_evt[6] = {0, 0, 0, 0, 0, 0};
  double regrid_evt_t[2] = {0.0, 0.0};
  // x3_ledger: outflow mass and count of the run, x3_removed (mass, count), dropped deposits
  double x3_outflow_mass = 0.0, x3_outflow_count = 0.0;
  double x3_removed[2] = {0.0, 0.0};
  std::vector<double> dropped_sum;
  // the cell-order index (status 1 stored, 2 omitted, 3 none; the cycle of the last sort)
  std::int32_t cloud_ord_status = 0;      // 0: no cloud_ord_n record
  std::int32_t cloud_ord_sort_cycle = -1;
  std::vector<std::int32_t> cloud_ord;
  std::vector<std::uint64_t> cloud_ord_tag;
  // records this build does not interpret, as read (name, bytes)
  std::vector<std::pair<std::string, std::vector<char>>> other;
};

// the section of np particles from host rows (row r of the reals at pr + r * stride)
std::string PackParticleRestartRows(const double *pr, const int *pi, long long stride,
                                    std::int64_t np, double dtnew,
                                    const ParticleRestartState &st, std::vector<char> &buf);

// the section of the particles of ctx (device rows copied on stream; synchronises)
std::string PackParticleRestart(const dustb_ctx &ctx, void *stream, double dtnew,
                                const ParticleRestartState &st, std::vector<char> &buf);

// a parsed section: rows in host vectors (nrdata x np, nidata x np; version 1 PTAGH = 0)
struct ParticleRestartSection {
  std::int32_t version = 0, ranks = 0, nrdata = 0, nidata = 0;
  std::int64_t np = 0;
  double dtnew = 0.0;
  std::vector<double> pr;
  std::vector<int> pi;   // always 5 rows
  ParticleRestartState state;
  std::vector<std::string> notes;   // unknown records, missing species table
};

// checks the section (magic at both ends, version, type sizes, a rank count of nsec, columns,
// sizes) and parses it (ParseSection + UnpackRestartState, src/dust/dust_restart.cpp)
std::string ParseParticleRestart(const std::vector<char> &buf, ParticleRestartSection &out,
                                 int nsec = 1);

// The particle sections of a restart file: a run on several ranks appends one section per
// rank, in rank order, each with "ranks written" in its head.  Splits file[at, end) into them
// by the byte count of each head (magic and size checked; the restart reader's section
// offsets, src/gravity/restart.cpp).
std::string SplitParticleRestart(const std::vector<char> &file, std::size_t at,
                                 std::vector<std::vector<char>> &sections);

// Whether rank `me` of a run on `nranks` ranks, holding blocks [gids, gids + nmb), can take
// its own section back exactly (UnpackParticleRestart, src/dust/dust_restart.cpp): as many
// sections as ranks and, with more than one, the section's rank_blocks record names this rank
// and these blocks.  A run on several ranks takes the exact path only when every rank's
// answer is yes (the reference reduces it with a logical and over the ranks).
std::string ParticleRestartOwnSectionMatches(const std::vector<std::vector<char>> &sections,
                                             int me, int nranks, int gids, int nmb,
                                             bool &match);

// The particles (and dust records) of rank `me`: exact (all ranks matched) -- its own
// section as written, every particle's PGID within its blocks (else an error: a particle
// names a MeshBlock that does not exist); otherwise the particles of its blocks from every
// section in section order, the records and dtnew of section 0, the tag counter unset (it
// starts again at the bound of all tags issued) and the cloud order index dropped (another
// layout: it is rebuilt).
std::string SelectParticleRestart(const std::vector<std::vector<char>> &sections, int me,
                                  int gids, int nmb, bool exact, ParticleRestartSection &out);

// the parsed rows into the device arrays of ctx (npart set to the section's; the capacity
// ctx.part.stride must hold them); synchronises
std::string RestoreParticleRows(const ParticleRestartSection &sec, dustb_ctx &ctx, void *stream);

}  // namespace athenak_b200

#endif  // ATHENAK_B200_RESTART_HPP_
