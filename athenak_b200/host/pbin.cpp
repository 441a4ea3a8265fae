// pbin.cpp -- the particle science file (src/outputs/pbin.cpp, ParticleBinaryOutput): the
// layout, the header and the compressed form; see pbin.hpp.
#include "pbin.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <iomanip>
#include <limits>
#include <sstream>
#include <thread>

#if ATHENAK_B200_HAVE_ZLIB
#include <zlib.h>
#endif

namespace athenak_b200 {
namespace {

constexpr char kMagic[9] = "AKPBIN01";
constexpr char kEnd[9] = "AKPBEND1";
constexpr std::uint32_t kVersion = 2, kVersionCompressed = 3;
constexpr std::uint64_t kAlign = 64, kPreamble = 64, kFooter = 16;

std::uint64_t Align(std::uint64_t a) { return a + (kAlign - a % kAlign) % kAlign; }

struct Col {
  std::string table, name, dtype, meaning;
  std::uint64_t itemsize = 0, count = 0, offset = 0, bytes = 0;
  int pcol = -1;                       // DUSTB_PBIN_* of a particle column
  bool encoded = false;                // version 3
  std::vector<unsigned char> stored;   // version 3: the chunks, concatenated
  std::vector<std::uint64_t> chunk_bytes;
};

std::uint64_t NumChunks(std::uint64_t n, std::uint64_t chunk_rows) {
  return (n == 0) ? 1 : (n - 1) / chunk_rows + 1;
}

int CompressThreads() {
  const unsigned h = std::thread::hardware_concurrency();
  return std::max(1, std::min(static_cast<int>(h ? h : 1), 32));
}

#if ATHENAK_B200_HAVE_ZLIB
// one complete zlib stream (RFC 1950), level 1
bool Deflate(const unsigned char *in, std::uint64_t bytes, std::vector<unsigned char> &out) {
  z_stream z;
  std::memset(&z, 0, sizeof(z));
  if (deflateInit(&z, 1) != Z_OK) return false;
  out.clear();
  std::vector<unsigned char> buf(std::size_t(1) << 18);
  const std::uint64_t piece = std::uint64_t(1) << 30;   // the zlib counters are 32-bit
  std::uint64_t done = 0;
  int flush = Z_NO_FLUSH, ret = Z_OK;
  do {
    const std::uint64_t nin = std::min(piece, bytes - done);
    z.next_in = const_cast<Bytef *>(in + done);
    z.avail_in = static_cast<uInt>(nin);
    done += nin;
    flush = (done == bytes) ? Z_FINISH : Z_NO_FLUSH;
    do {
      z.next_out = buf.data();
      z.avail_out = static_cast<uInt>(buf.size());
      ret = deflate(&z, flush);
      if (ret == Z_STREAM_ERROR) { deflateEnd(&z); return false; }
      out.insert(out.end(), buf.data(), buf.data() + (buf.size() - z.avail_out));
    } while (z.avail_out == 0);
  } while (flush != Z_FINISH);
  deflateEnd(&z);
  return ret == Z_STREAM_END;
}
#endif

// version 3: the chunks of one column (n rows of size bytes), shuffled here unless the bytes
// come shuffled, deflated by a pool of threads; chunk order and bytes do not depend on the
// thread count
bool ShuffleDeflate(const unsigned char *src, std::uint64_t n, std::uint64_t size,
                    std::uint64_t chunk_rows, bool shuffled, Col &c) {
  const std::uint64_t nchunk = NumChunks(n, chunk_rows);
  c.stored.clear();
  c.chunk_bytes.assign(nchunk, 0);
  if (n == 0) return true;
#if ATHENAK_B200_HAVE_ZLIB
  std::vector<std::vector<unsigned char>> part(nchunk);
  std::atomic<std::uint64_t> next(0);
  std::atomic<int> failed(0);
  auto work = [&]() {
    std::vector<unsigned char> sh;
    for (std::uint64_t j = next++; j < nchunk; j = next++) {
      const std::uint64_t r0 = j * chunk_rows, rows = std::min(chunk_rows, n - r0);
      const unsigned char *in = src + r0 * size;
      if (!shuffled && size > 1) {
        sh.resize(static_cast<std::size_t>(rows * size));
        for (std::uint64_t k = 0; k < size; ++k)
          for (std::uint64_t i = 0; i < rows; ++i) sh[k * rows + i] = in[i * size + k];
        in = sh.data();
      }
      if (!Deflate(in, rows * size, part[j])) failed = 1;
      c.chunk_bytes[j] = part[j].size();
    }
  };
  std::vector<std::thread> pool;
  const int nt = static_cast<int>(std::min<std::uint64_t>(CompressThreads(), nchunk));
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto &t : pool) t.join();
  if (failed) return false;
  std::uint64_t total = 0;
  for (const auto &p : part) total += p.size();
  c.stored.resize(static_cast<std::size_t>(total));
  std::uint64_t at = 0;
  for (auto &p : part) {
    if (!p.empty()) std::memcpy(c.stored.data() + at, p.data(), p.size());
    at += p.size();
    std::vector<unsigned char>().swap(p);
  }
  return true;
#else
  (void)src; (void)size; (void)shuffled;
  return false;
#endif
}

bool LittleEndian() {
  const std::uint32_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

bool WriteBytes(std::FILE *f, const void *p, std::uint64_t n) {
  return n == 0 || std::fwrite(p, 1, static_cast<std::size_t>(n), f) == n;
}

bool WriteZeros(std::FILE *f, std::uint64_t n) {
  static const unsigned char z[64] = {0};
  while (n > 0) {
    const std::uint64_t k = std::min<std::uint64_t>(n, sizeof(z));
    if (std::fwrite(z, 1, static_cast<std::size_t>(k), f) != k) return false;
    n -= k;
  }
  return true;
}

}  // namespace

bool PbinCanCompress() { return ATHENAK_B200_HAVE_ZLIB != 0; }

bool PbinPlan::has(int column) const {
  if (column == DUSTB_PBIN_SPECIES || column == DUSTB_PBIN_STOPPING_TIME) return !constant_sp_ts;
  if (column == DUSTB_PBIN_MASS) return !constant_mass;
  return column >= DUSTB_PBIN_ID && column <= DUSTB_PBIN_STOPPING_TIME;
}

PbinPlan PlanPbin(const PbinMeta &meta, const dustb_pbin_stats &st) {
  PbinPlan p;
  p.ts0 = meta.taus.empty() ? 0.0 : meta.taus[0];
  p.constant_sp_ts = meta.nspecies == 1 && meta.stopping_time_mode == "species_fixed" &&
                     !meta.taus.empty() && st.differ_rows == 0;
  p.constant_mass = st.active_rows > 0 && st.invalid_mass_rows == 0 &&
                    st.mass_min == st.mass_max;
  p.mass = st.mass_min;
  return p;
}

std::string PbinFileName(const std::string &dir, const PbinMeta &meta) {
  char number[16];
  std::snprintf(number, sizeof(number), "%05d", meta.file_number);
  return dir + "/pbin/" + meta.basename + "." + meta.file_id + "." + number + ".pbin";
}

std::uint64_t PbinTopologyHash(const std::vector<PbinBlock> &blocks) {
  // FNV-1a with the 64-bit prime 1099511628211 and the format's start value
  // 1469598103934665603 (the value the pbin readers compare against; it is not the usual
  // FNV offset basis)
  std::uint64_t h = 1469598103934665603ULL;
  for (const auto &b : blocks) {
    const std::int64_t v[4] = {b.level, b.lx1, b.lx2, b.lx3};
    for (int q = 0; q < 4; ++q)
      for (int k = 0; k < 8; ++k) {
        h ^= (static_cast<std::uint64_t>(v[q]) >> (8 * k)) & 0xffu;
        h *= 1099511628211ULL;
      }
  }
  return h;
}

std::string WritePbinFile(const std::string &path, const PbinMeta &meta,
                          const dustb_pbin_stats &st, const PbinRows &rows,
                          const std::vector<PbinBlock> &blocks) {
  if (meta.compress && !PbinCanCompress()) return "pbin: version 3 needs zlib (built without it)";
  if (meta.compress && meta.chunk_rows < 1) return "pbin: chunk_rows must be positive";
  if (rows.n != static_cast<std::uint64_t>(st.active_rows)) return "pbin: row count mismatch";
  const bool little = LittleEndian();
  const std::string bo = little ? "<" : ">";
  const PbinPlan plan = PlanPbin(meta, st);
  const std::uint64_t ntotal = rows.n, nblocks = blocks.size();
  const char *rdt = meta.single_precision ? "f4" : "f8";
  const std::uint64_t rsz = meta.single_precision ? 4 : 8;
  const std::uint32_t version = meta.compress ? kVersionCompressed : kVersion;

  // ---- the columns, in the reference's order
  std::vector<Col> cols;
  auto col = [&](const char *table, const char *name, const char *dt, std::uint64_t size,
                 const std::string &meaning, int pcol) {
    Col c;
    c.table = table; c.name = name; c.dtype = bo + dt; c.itemsize = size; c.meaning = meaning;
    c.count = (c.table == "particles") ? ntotal : nblocks;
    c.pcol = pcol;
    cols.push_back(c);
  };
  const char *species_meaning = "species_id (0-based; input index N = species_id + 1)";
  const char *ts_meaning = "stopping time t_s (code time)";
  const char *mass_meaning = "macro-particle mass (code units; not a grain mass)";
  col("particles", "id", "u8", 8, "numerical sample identity: the 64-bit tag; split / merge / "
      "resampling create and remove samples, an id is not a grain lineage", DUSTB_PBIN_ID);
  if (!plan.constant_sp_ts) col("particles", "species", "u4", 4, species_meaning, DUSTB_PBIN_SPECIES);
  col("particles", "x1", rdt, rsz, "position x1 (code length)", DUSTB_PBIN_X1);
  col("particles", "x2", rdt, rsz, "position x2 (code length)", DUSTB_PBIN_X2);
  col("particles", "x3", rdt, rsz, meta.ndim == 3 ? "position x3 (code length)" :
      "x3 column of a 2-D run (not a mesh direction; as stored)", DUSTB_PBIN_X3);
  col("particles", "v1", rdt, rsz, "velocity component 1 (see [frame])", DUSTB_PBIN_V1);
  col("particles", "v2", rdt, rsz, "velocity component 2 (see [frame])", DUSTB_PBIN_V2);
  col("particles", "v3", rdt, rsz, "velocity component 3 (see [frame])", DUSTB_PBIN_V3);
  if (!plan.constant_mass) col("particles", "mass", rdt, rsz, mass_meaning, DUSTB_PBIN_MASS);
  if (!plan.constant_sp_ts)
    col("particles", "stopping_time", rdt, rsz, ts_meaning, DUSTB_PBIN_STOPPING_TIME);
  col("blocks", "gid", "i8", 8, "MeshBlock global id", -1);
  col("blocks", "rank", "i4", 4, "MPI rank that wrote the block", -1);
  col("blocks", "level", "i4", 4, "refinement level above the root level", -1);
  col("blocks", "lx1", "i8", 8, "logical location x1 (at the block's level)", -1);
  col("blocks", "lx2", "i8", 8, "logical location x2", -1);
  col("blocks", "lx3", "i8", 8, "logical location x3", -1);
  col("blocks", "x1min", "f8", 8, "block box x1min", -1);
  col("blocks", "x1max", "f8", 8, "block box x1max", -1);
  col("blocks", "x2min", "f8", 8, "block box x2min", -1);
  col("blocks", "x2max", "f8", 8, "block box x2max", -1);
  col("blocks", "x3min", "f8", 8, "block box x3min", -1);
  col("blocks", "x3max", "f8", 8, "block box x3max", -1);

  // ---- version 3: every particle column compressed first (the stored sizes set the layout)
  std::vector<unsigned char> buf;
  std::uint64_t raw_bytes = 0, stored_bytes = 0;
  if (meta.compress) {
    for (auto &c : cols) {
      if (c.pcol < 0) continue;
      c.encoded = true;
      if (ntotal > 0) {
        buf.clear();
        if (!rows.fetch || !rows.fetch(c.pcol, c.itemsize, buf) ||
            buf.size() != ntotal * c.itemsize)
          return "pbin: column " + c.name + " not available";
      }
      if (!ShuffleDeflate(buf.data(), ntotal, c.itemsize, meta.chunk_rows, rows.shuffled, c))
        return "pbin: zlib deflate failed (column " + c.name + ")";
    }
  }
  std::uint64_t at = 0;
  for (auto &c : cols) {
    c.offset = at;
    if (c.encoded) {
      c.bytes = c.stored.size();
      raw_bytes += c.count * c.itemsize;
      stored_bytes += c.bytes;
    } else {
      c.bytes = c.count * c.itemsize;
    }
    at = Align(at + c.bytes);
  }
  const std::uint64_t data_bytes = at;

  // ---- the text header
  std::ostringstream h;
  h << std::setprecision(17);
  h << "AthenaK particle science file (pbin) format_version = " << version << "\n";
  h << "[file]\n";
  h << "format = AKPBIN\nformat_version = " << version << "\n";
  if (meta.compress) h << "encoding = shuffle_deflate  # particle columns compressed, see [encoding]\n";
  h << "byte_order = " << (little ? "little" : "big") << "\n";
  h << "n_particles = " << ntotal << "\nn_blocks = " << nblocks << "\n";
  h << "written_by_ranks = 1\n";
  h << "completeness = footer AKPBEND1 + file size; written as .tmp, renamed when complete\n";
  h << "[snapshot]\n";
  h << "time = " << meta.time << "\ncycle = " << meta.cycle << "\n";
  h << "dt = " << meta.dt << "\n";
  h << "basename = " << meta.basename << "\n";
  h << "output_block = " << meta.block_name << "\n";
  h << "file_number = " << meta.file_number << "\n";
  h << "source_commit = " << meta.source_commit << "\n";
  h << "mesh_update_seq = " << meta.mesh_update_seq << "\n";
  {
    std::ostringstream hx;
    hx << "0x" << std::hex << std::setw(16) << std::setfill('0') << PbinTopologyHash(blocks);
    h << "block_topology_hash = " << hx.str() << "  # FNV-1a 64 of (level, lx1, lx2, lx3) "
      << "as int64 for every block in gid order\n";
  }
  h << "output_point = end of a cycle, before that cycle's mesh refinement check (the first "
    << "output: after the problem generator; the last: after the final check)\n";
  h << "[mesh]\n";
  h << "ndim = " << meta.ndim << "\n";
  h << "nx1 = " << meta.nx1 << "\nnx2 = " << meta.nx2 << "\nnx3 = " << meta.nx3 << "\n";
  h << "x1min = " << meta.x1min << "\nx1max = " << meta.x1max << "\n";
  h << "x2min = " << meta.x2min << "\nx2max = " << meta.x2max << "\n";
  h << "x3min = " << meta.x3min << "\nx3max = " << meta.x3max << "\n";
  h << "meshblock_nx1 = " << meta.mb_nx1 << "\nmeshblock_nx2 = " << meta.mb_nx2
    << "\nmeshblock_nx3 = " << meta.mb_nx3 << "\n";
  h << "levels = " << meta.levels << "  # finest level above the root\n";
  h << "multilevel = " << meta.multilevel << "\nadaptive = " << meta.adaptive << "\n";
  const char *face[6] = {"ix1", "ox1", "ix2", "ox2", "ix3", "ox3"};
  for (int f = 0; f < 6; ++f) h << "bc_" << face[f] << " = " << meta.bc[f] << "\n";
  h << "[particles]\n";
  h << "rows = active rows only (the capacity tail and zero-mass rows are left out)\n";
  h << "row_order = by writing rank, then the rank's array order (unsorted; neither the "
    << "order nor the rank layout is stable between outputs)\n";
  h << "zero_mass_rows_excluded = " << st.zero_mass_rows << "\n";
  h << "invalid_mass_rows = " << st.invalid_mass_rows << "  # negative or non-finite mass "
    << "(written)\n";
  h << "negative_tag_rows = " << st.negative_tag_rows << "  # tags >= 2^63 (high word below "
    << "zero; never issued; the key keeps its version-1 name)\n";
  h << "owner = not stored: the MeshBlock whose half-open box [min, max) holds the position "
    << "(blocks table)\n";
  {
    std::string names;
    if (plan.constant_sp_ts) names += "species stopping_time";
    if (plan.constant_mass) names += std::string(names.empty() ? "" : " ") + "mass";
    h << "constant_columns = " << (names.empty() ? std::string("none") : names);
    if (!names.empty()) h << "  # the same value in every row, given in [constants]";
    const bool sp_candidate = meta.nspecies == 1 && meta.stopping_time_mode == "species_fixed" &&
                              !meta.taus.empty();
    if (sp_candidate && !plan.constant_sp_ts && st.differ_rows > 0)
      h << (names.empty() ? "  # " : "; ") << "one species, species_fixed, but " << st.differ_rows
        << " rows differ from species 0 / its tau_s: kept as columns";
    h << "\n";
  }
  h << "particle_real_precision = " << (meta.single_precision ? "single" : "double")
    << "  # positions, velocities, mass, stopping time (<outputN>/precision)\n";
  h << "[species]\n";
  h << "nspecies = " << meta.nspecies << "\n";
  h << "stopping_time_mode = " << meta.stopping_time_mode << "  # stopping_time (column or "
    << "constant) is the value each particle uses\n";
  if (meta.legacy_species) {
    h << "dust_to_gas = " << meta.dust_to_gas << "  # the <dust>/dust_to_gas key only; a "
      << "problem generator may set its own abundances (e.g. <problem>/eps_N, see [input])\n";
  }
  h << "back_reaction = " << meta.back_reaction << "\n";
  for (const auto &line : meta.species_table) h << line << "\n";
  for (int s = 0; s < meta.nspecies; ++s) {
    h << "species." << s << " = input_index " << (s + 1) << ", tau_s "
      << (s < static_cast<int>(meta.taus.size()) ? meta.taus[s]
                                                 : std::numeric_limits<double>::quiet_NaN());
    if (s < static_cast<int>(meta.species_detail.size())) h << meta.species_detail[s];
    h << "\n";
  }
  h << "[representation]\n";
  for (const auto &line : meta.representation) h << line << "\n";
  h << "[frame]\n";
  h << "positions = lab frame, code length\n";
  if (meta.shearing_box) {
    h << "velocity_frame = shear_relative  # velocities relative to the background shear "
      << "-q Omega x1\n";
    h << "shear_q = " << meta.qshear << "\nshear_omega = " << meta.omega0 << "\n";
    if (meta.ndim == 3) {
      h << "axes = x1 radial, x2 azimuthal, x3 vertical\n";
      h << "azimuthal_velocity = v2  # v2_phys = v2 - q*Omega*x1\n";
    } else {
      h << "axes = x1 radial, x2 vertical (2-D r-z shearing box), azimuth not a mesh "
        << "direction\n";
      h << "azimuthal_velocity = v3  # v3_phys = v3 - q*Omega*x1; v2 is vertical\n";
    }
  } else {
    h << "velocity_frame = lab\n";
  }
  if (meta.compress) {
    h << "[encoding]\n";
    h << "particle_columns = shuffle_deflate  # every particles column; the blocks columns "
      << "are raw\n";
    h << "chunk_rows = " << meta.chunk_rows << "  # rows per chunk at most; a chunk holds rows "
      << "of one writing rank\n";
    h << "shuffle = byte shuffle per chunk: stored[k*rows + i] = raw[i*itemsize + k] for "
      << "byte k = 0 .. itemsize-1 of row i (raw bytes in the file byte order)\n";
    h << "deflate = one complete zlib stream per chunk (RFC 1950: deflate + adler32), "
      << "level 1\n";
    h << "chunk_layout = the chunks of a column follow one another without padding, by "
      << "rank, then by row; a rank without rows has one chunk with rows 0 and "
      << "stored_bytes 0\n";
    h << "chunk_table = [chunks]  # chunk = column rank first_row rows offset stored_bytes; "
      << "raw bytes = rows * itemsize\n";
    h << "particle_raw_bytes = " << raw_bytes << "\n";
    h << "particle_stored_bytes = " << stored_bytes << "\n";
  }
  h << "[columns]\n";
  if (meta.compress) {
    h << "# column = table name dtype count offset bytes encoding (offset from data_start; "
      << "bytes stored: count * itemsize when raw)\n";
  } else {
    h << "# column = table name dtype count offset bytes (offset from data_start)\n";
  }
  for (const auto &c : cols) {
    h << "column = " << c.table << " " << c.name << " " << c.dtype << " " << c.count << " "
      << c.offset << " " << c.bytes;
    if (meta.compress) h << (c.encoded ? " shuffle_deflate" : " raw");
    h << "\n";
  }
  if (meta.compress) {
    h << "[chunks]\n";
    h << "# chunk = column rank first_row rows offset stored_bytes (offset from "
      << "data_start)\n";
    for (const auto &c : cols) {
      if (!c.encoded) continue;
      std::uint64_t off = c.offset, row = 0;
      const std::uint64_t nch = NumChunks(ntotal, meta.chunk_rows);
      for (std::uint64_t j = 0; j < nch; ++j) {
        const std::uint64_t r = (ntotal == 0) ? 0 : std::min(meta.chunk_rows, ntotal - j * meta.chunk_rows);
        const std::uint64_t sb = c.chunk_bytes[j];
        h << "chunk = " << c.name << " 0 " << row << " " << r << " " << off << " " << sb << "\n";
        off += sb;
        row += r;
      }
    }
  }
  h << "[constants]\n";
  h << "# constant = table name dtype value (the same value in every row of the table)\n";
  if (plan.constant_sp_ts) {
    h << "constant = particles species " << bo << "u4 0\n";
    h << "constant = particles stopping_time " << bo << "f8 " << plan.ts0 << "\n";
  }
  if (plan.constant_mass) h << "constant = particles mass " << bo << "f8 " << plan.mass << "\n";
  h << "[meaning]\n";
  for (const auto &c : cols) h << c.table << "." << c.name << " = " << c.meaning << "\n";
  if (plan.constant_sp_ts) {
    h << "particles.species = " << species_meaning << "\n";
    h << "particles.stopping_time = " << ts_meaning << "\n";
  }
  if (plan.constant_mass) h << "particles.mass = " << mass_meaning << "\n";
  h << "[input]\n";
  h << meta.input_dump;
  const std::string text = h.str();
  const std::uint64_t data_start = Align(kPreamble + text.size());
  const std::uint64_t file_bytes = data_start + data_bytes + kFooter;

  // ---- the file, as <path>.tmp, renamed when complete
  const std::string tmp = path + ".tmp";
  std::FILE *f = std::fopen(tmp.c_str(), "wb");
  if (!f) return "pbin: cannot open " + tmp;
  bool ok = true;
  {
    unsigned char pre[kPreamble] = {0};
    std::memcpy(pre, kMagic, 8);
    const std::uint32_t mark = 0x01020304u;
    std::memcpy(pre + 8, &mark, 4);
    std::memcpy(pre + 12, &version, 4);
    const std::uint64_t v[6] = {text.size(), data_start, data_bytes, ntotal, nblocks, 0};
    std::memcpy(pre + 16, v, sizeof(v));
    ok = WriteBytes(f, pre, kPreamble) && WriteBytes(f, text.data(), text.size()) &&
         WriteZeros(f, data_start - kPreamble - text.size());
  }
  std::vector<std::int64_t> i8(blocks.size());
  std::vector<std::int32_t> i4(blocks.size());
  std::vector<double> f8(blocks.size());
  for (const auto &c : cols) {
    if (!ok) break;
    const void *src = nullptr;
    if (c.encoded) {
      src = c.stored.data();
    } else if (c.pcol >= 0) {
      if (ntotal > 0) {
        buf.clear();
        if (!rows.fetch || rows.shuffled || !rows.fetch(c.pcol, c.itemsize, buf) ||
            buf.size() != c.bytes) {
          std::fclose(f);
          std::remove(tmp.c_str());
          return "pbin: column " + c.name + " not available";
        }
        src = buf.data();
      }
    } else {
      for (std::size_t m = 0; m < blocks.size(); ++m) {
        const PbinBlock &b = blocks[m];
        if (c.name == "gid") i8[m] = b.gid;
        if (c.name == "rank") i4[m] = b.rank;
        if (c.name == "level") i4[m] = b.level;
        if (c.name == "lx1") i8[m] = b.lx1;
        if (c.name == "lx2") i8[m] = b.lx2;
        if (c.name == "lx3") i8[m] = b.lx3;
        if (c.name == "x1min") f8[m] = b.x1min;
        if (c.name == "x1max") f8[m] = b.x1max;
        if (c.name == "x2min") f8[m] = b.x2min;
        if (c.name == "x2max") f8[m] = b.x2max;
        if (c.name == "x3min") f8[m] = b.x3min;
        if (c.name == "x3max") f8[m] = b.x3max;
      }
      src = (c.dtype == bo + "i8") ? static_cast<const void *>(i8.data())
            : (c.dtype == bo + "i4") ? static_cast<const void *>(i4.data())
                                     : static_cast<const void *>(f8.data());
    }
    ok = WriteBytes(f, src, c.bytes) && WriteZeros(f, Align(c.offset + c.bytes) - c.offset - c.bytes);
  }
  if (ok) {
    unsigned char foot[kFooter];
    std::memcpy(foot, kEnd, 8);
    std::memcpy(foot + 8, &file_bytes, 8);
    ok = WriteBytes(f, foot, kFooter);
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { std::remove(tmp.c_str()); return "pbin: write failed on " + tmp; }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) return "pbin: could not rename " + tmp;
  return "";
}

std::string WriteParticleBinary(const dustb_ctx &ctx, void *stream, const std::string &path,
                                const PbinMeta &meta, const std::vector<PbinBlock> &blocks,
                                dustb_pbin_stats *stats_out) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int np = ctx.part.npart;
  const long long sbytes = dustb_pbin_scratch_bytes(np);
  void *scratch = nullptr, *dbuf = nullptr, *dshuf = nullptr;
  int *idx = nullptr;
  dustb_pbin_stats *dst = nullptr;
  std::string err;
  auto fail = [&](const std::string &e) {
    if (err.empty()) err = e;
  };
  if (cudaMalloc(&scratch, (size_t)sbytes) != cudaSuccess ||
      cudaMalloc(&idx, sizeof(int) * (size_t)std::max(np, 1)) != cudaSuccess ||
      cudaMalloc(&dst, sizeof(dustb_pbin_stats)) != cudaSuccess)
    fail("pbin: device scratch not allocated");
  dustb_pbin_stats hs{};
  if (err.empty()) {
    const double ts0 = meta.taus.empty() ? 0.0 : meta.taus[0];
    if (dustb_pbin_rows(&ctx, idx, dst, ts0, scratch, sbytes, stream) != DUSTB_OK)
      fail(std::string("pbin: ") + dustb_last_error());
    else if (cudaMemcpyAsync(&hs, dst, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
             cudaStreamSynchronize(st) != cudaSuccess)
      fail("pbin: row statistics not read");
  }
  const std::uint64_t n = static_cast<std::uint64_t>(hs.active_rows);
  if (err.empty() && n > 0 &&
      (cudaMalloc(&dbuf, (size_t)(n * 8)) != cudaSuccess ||
       (meta.compress && cudaMalloc(&dshuf, (size_t)(n * 8)) != cudaSuccess)))
    fail("pbin: device column buffer not allocated");
  if (err.empty()) {
    PbinRows rows;
    rows.n = n;
    rows.shuffled = meta.compress;
    rows.fetch = [&](int column, std::uint64_t itemsize, std::vector<unsigned char> &out) {
      const int single = (itemsize == 4 && column >= DUSTB_PBIN_X1) ? 1 : 0;
      if (dustb_pbin_pack(&ctx, idx, (int)n, column, single, dbuf, stream) != DUSTB_OK) return false;
      const void *src = dbuf;
      if (meta.compress) {
        if (dustb_pbin_shuffle(dbuf, (long long)n, (int)itemsize, (long long)meta.chunk_rows,
                               dshuf, stream) != DUSTB_OK)
          return false;
        src = dshuf;
      }
      out.resize((size_t)(n * itemsize));
      return cudaMemcpyAsync(out.data(), src, out.size(), cudaMemcpyDeviceToHost, st) ==
                 cudaSuccess &&
             cudaStreamSynchronize(st) == cudaSuccess;
    };
    err = WritePbinFile(path, meta, hs, rows, blocks);
  }
  if (stats_out) *stats_out = hs;
  cudaFree(scratch); cudaFree(idx); cudaFree(dst); cudaFree(dbuf); cudaFree(dshuf);
  return err;
}

}  // namespace athenak_b200
