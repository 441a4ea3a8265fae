// pbin.hpp -- the particle science file (file_type = pbin) of the dust particles, written as
// ParticleBinaryOutput writes it (src/outputs/pbin.cpp): a 64-byte preamble, the text header
// ([file] [snapshot] [mesh] [particles] [species] [representation] [frame] ([encoding]
// [chunks] in version 3) [columns] [constants] [input]), the columns one after the
// other at 64-byte boundaries, the footer "AKPBEND1" + file size; written as <name>.tmp and
// renamed when complete.  Only the active rows (mass != 0) are written; species and stopping
// time, and the mass, become header constants under the reference's conditions.  Format
// version 2 stores the columns raw; version 3 (compress) stores every particle column
// byte-shuffled and deflated (zlib level 1) in chunks of chunk_rows rows.
//
// One rank writes the whole file (the reference's MPI-IO prefix offsets reduce to rank 0's).
// The device side (the active rows, the column packing, the byte shuffle) is in the C ABI
// (dustb_pbin_*); WriteParticleBinary drives it, WritePbinFile writes host columns.
#ifndef ATHENAK_B200_PBIN_HPP_
#define ATHENAK_B200_PBIN_HPP_

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "../../include/dustb.h"

namespace athenak_b200 {

// one MeshBlock of the blocks table (gid order)
struct PbinBlock {
  std::int64_t gid = 0, lx1 = 0, lx2 = 0, lx3 = 0;
  std::int32_t rank = 0, level = 0;   // level above the root
  double x1min = 0, x1max = 0, x2min = 0, x2max = 0, x3min = 0, x3max = 0;
};

// what the header says about the run (the reference reads these from the Mesh, the
// DustGasDrag and the ParameterInput)
struct PbinMeta {
  // [snapshot] and the file name pbin/<basename>.<file_id>.<NNNNN>.pbin
  double time = 0.0, dt = 0.0;
  long long cycle = 0;
  std::string basename = "dust", block_name = "output2", file_id = "particles";
  int file_number = 0;
  std::string source_commit = "unknown";
  long long mesh_update_seq = 0;
  // [mesh]
  int ndim = 3;
  int nx1 = 1, nx2 = 1, nx3 = 1, mb_nx1 = 1, mb_nx2 = 1, mb_nx3 = 1;
  double x1min = 0, x1max = 1, x2min = 0, x2max = 1, x3min = 0, x3max = 1;
  int levels = 0, multilevel = 0, adaptive = 0;
  std::string bc[6] = {"periodic", "periodic", "periodic", "periodic", "periodic", "periodic"};
  // [species]
  int nspecies = 1;
  std::string stopping_time_mode = "species_fixed";   // or particle_static, dynamic
  std::vector<double> taus;                           // tau_s of each species
  bool legacy_species = true;                         // the dust_to_gas line (no new init)
  double dust_to_gas = 0.0;
  int back_reaction = 1;
  std::vector<std::string> species_table;   // SpeciesTable::Describe lines after nspecies
  std::vector<std::string> species_detail;  // per species: text after "tau_s <value>"
  // [representation]: DustGasDrag::ScienceRepresentation lines
  std::vector<std::string> representation = {"particles = point  # point particles"};
  // [frame]
  bool shearing_box = false;
  double qshear = 1.5, omega0 = 1.0;
  // <outputN> options: precision = single; test_pbin_compress; test_pbin_chunk_rows
  bool single_precision = false;
  bool compress = false;
  std::uint64_t chunk_rows = std::uint64_t(1) << 20;
  // [input]: the parameter dump
  std::string input_dump = "<par_end>\n";
};

// the active rows' columns, one at a time: fetch(column, itemsize, bytes) fills bytes with
// the n values of particle column DUSTB_PBIN_* (itemsize 4 or 8), raw or, with shuffled,
// already byte-shuffled chunk by chunk (dustb_pbin_shuffle; version 3 only); false on error
struct PbinRows {
  std::uint64_t n = 0;
  std::function<bool(int, std::uint64_t, std::vector<unsigned char> &)> fetch;
  bool shuffled = false;
};

// which particle columns the file holds (the reference's version 2 rules)
struct PbinPlan {
  bool constant_sp_ts = false, constant_mass = false;
  double ts0 = 0.0, mass = 0.0;
  bool has(int column) const;
};
PbinPlan PlanPbin(const PbinMeta &meta, const dustb_pbin_stats &stats);

// the file name pbin/<basename>.<file_id>.<NNNNN>.pbin under dir
std::string PbinFileName(const std::string &dir, const PbinMeta &meta);

// writes the file; returns "" on success, else the error
std::string WritePbinFile(const std::string &path, const PbinMeta &meta,
                          const dustb_pbin_stats &stats, const PbinRows &rows,
                          const std::vector<PbinBlock> &blocks);

// the whole output from the device arrays of ctx on stream: the active rows and their columns
// (packed, and shuffled for version 3, on the device), then WritePbinFile.  Synchronises.
std::string WriteParticleBinary(const dustb_ctx &ctx, void *stream, const std::string &path,
                                const PbinMeta &meta, const std::vector<PbinBlock> &blocks,
                                dustb_pbin_stats *stats_out = nullptr);

// FNV-1a 64 over (level, lx1, lx2, lx3) of every block as little-endian int64, from the
// format's start value
std::uint64_t PbinTopologyHash(const std::vector<PbinBlock> &blocks);

// whether this build writes version 3 (zlib present)
bool PbinCanCompress();

}  // namespace athenak_b200

#endif  // ATHENAK_B200_PBIN_HPP_
