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
  std::string table, name, dtype;
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
// the zlib stream (RFC 1950: deflate data and its adler32) of one chunk at level 1, made by
// zlib's one-shot compressor into a buffer of its worst-case size
bool ZlibChunk(const unsigned char *in, std::uint64_t n, std::vector<unsigned char> &out) {
  uLongf cap = compressBound(static_cast<uLong>(n));
  out.resize(static_cast<std::size_t>(cap));
  if (compress2(out.data(), &cap, in, static_cast<uLong>(n), 1) != Z_OK) return false;
  out.resize(static_cast<std::size_t>(cap));
  return true;
}
#endif

// Version 3: column c of n rows of `size` bytes as consecutive chunks of at most chunk_rows
// rows, each byte-shuffled (byte k of row i to position k * rows + i; skipped when the rows
// arrive shuffled already) and compressed on its own.  Thread t of the pool takes chunks
// t, t + T, t + 2T, ...; the stored bytes are the chunks in row order, whatever T is.
bool EncodeColumn(const unsigned char *src, std::uint64_t n, std::uint64_t size,
                  std::uint64_t chunk_rows, bool pre_shuffled, Col &c) {
  const std::uint64_t nchunk = NumChunks(n, chunk_rows);
  c.stored.clear();
  c.chunk_bytes.assign(nchunk, 0);
  if (n == 0) return true;
#if ATHENAK_B200_HAVE_ZLIB
  std::vector<std::vector<unsigned char>> enc(nchunk);
  const int nthread = static_cast<int>(std::min<std::uint64_t>(CompressThreads(), nchunk));
  std::vector<char> good(nthread, 1);
  auto encode = [&](int t) {
    std::vector<unsigned char> shuffled;
    for (std::uint64_t j = t; j < nchunk; j += nthread) {
      const std::uint64_t first = j * chunk_rows;
      const std::uint64_t rows = std::min(chunk_rows, n - first);
      const unsigned char *rowbytes = src + first * size;
      if (!pre_shuffled && size > 1) {
        shuffled.resize(static_cast<std::size_t>(rows * size));
        for (std::uint64_t i = 0; i < rows; ++i)
          for (std::uint64_t k = 0; k < size; ++k) shuffled[k * rows + i] = rowbytes[i * size + k];
        rowbytes = shuffled.data();
      }
      if (!ZlibChunk(rowbytes, rows * size, enc[j])) good[t] = 0;
    }
  };
  std::vector<std::thread> helpers;
  for (int t = 1; t < nthread; ++t) helpers.emplace_back(encode, t);
  encode(0);
  for (auto &h : helpers) h.join();
  for (char g : good)
    if (!g) return false;
  std::uint64_t total = 0;
  for (std::uint64_t j = 0; j < nchunk; ++j) {
    c.chunk_bytes[j] = enc[j].size();
    total += enc[j].size();
  }
  c.stored.reserve(static_cast<std::size_t>(total));
  for (auto &e : enc) {
    c.stored.insert(c.stored.end(), e.begin(), e.end());
    std::vector<unsigned char>().swap(e);
  }
  return true;
#else
  (void)src; (void)size; (void)pre_shuffled;
  return false;
#endif
}

// the text header, section by section: "[name]" lines and "key = value" lines, an optional
// note after "  # " (readers drop it)
class HeaderText {
 public:
  HeaderText() { o_ << std::setprecision(17); }
  void line(const std::string &l) { o_ << l << "\n"; }
  void section(const char *name) { o_ << "[" << name << "]\n"; }
  template <class T>
  void key(const std::string &k, const T &v, const char *note = nullptr) {
    o_ << k << " = " << v;
    if (note) o_ << "  # " << note;
    o_ << "\n";
  }
  void raw(const std::string &text) { o_ << text; }
  std::string str() const { return o_.str(); }

 private:
  std::ostringstream o_;
};

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

  // ---- the column directory: the particle columns the plan keeps, then the blocks table
  std::vector<Col> cols;
  auto add = [&](const char *table, const char *name, const char *dt, std::uint64_t size,
                 int pcol) {
    Col c;
    c.table = table; c.name = name; c.dtype = bo + dt; c.itemsize = size; c.pcol = pcol;
    c.count = (c.table == "particles") ? ntotal : nblocks;
    cols.push_back(c);
  };
  add("particles", "id", "u8", 8, DUSTB_PBIN_ID);
  if (!plan.constant_sp_ts) add("particles", "species", "u4", 4, DUSTB_PBIN_SPECIES);
  add("particles", "x1", rdt, rsz, DUSTB_PBIN_X1);
  add("particles", "x2", rdt, rsz, DUSTB_PBIN_X2);
  add("particles", "x3", rdt, rsz, DUSTB_PBIN_X3);
  add("particles", "v1", rdt, rsz, DUSTB_PBIN_V1);
  add("particles", "v2", rdt, rsz, DUSTB_PBIN_V2);
  add("particles", "v3", rdt, rsz, DUSTB_PBIN_V3);
  if (!plan.constant_mass) add("particles", "mass", rdt, rsz, DUSTB_PBIN_MASS);
  if (!plan.constant_sp_ts) add("particles", "stopping_time", rdt, rsz, DUSTB_PBIN_STOPPING_TIME);
  for (const char *n : {"gid", "lx1", "lx2", "lx3"}) add("blocks", n, "i8", 8, -1);
  for (const char *n : {"rank", "level"}) add("blocks", n, "i4", 4, -1);
  for (const char *n : {"x1min", "x1max", "x2min", "x2max", "x3min", "x3max"})
    add("blocks", n, "f8", 8, -1);

  // ---- version 3: the particle columns are encoded first (their stored sizes place them)
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
      if (!EncodeColumn(buf.data(), ntotal, c.itemsize, meta.chunk_rows, rows.shuffled, c))
        return "pbin: compression failed (column " + c.name + ")";
    }
  }
  std::uint64_t at = 0;
  for (auto &c : cols) {
    c.offset = at;
    c.bytes = c.encoded ? c.stored.size() : c.count * c.itemsize;
    if (c.encoded) { raw_bytes += c.count * c.itemsize; stored_bytes += c.bytes; }
    at = Align(at + c.bytes);
  }
  const std::uint64_t data_bytes = at;

  // ---- the text header: what the readers parse, in the format's sections and key names
  HeaderText h;
  h.line("AthenaK particle science file (pbin) format_version = " + std::to_string(version));
  h.section("file");
  h.key("format", "AKPBIN");
  h.key("format_version", version);
  if (meta.compress) h.key("encoding", "shuffle_deflate");
  h.key("byte_order", little ? "little" : "big");
  h.key("n_particles", ntotal);
  h.key("n_blocks", nblocks);
  h.key("written_by_ranks", 1);
  h.section("snapshot");
  h.key("time", meta.time);
  h.key("cycle", meta.cycle);
  h.key("dt", meta.dt);
  h.key("basename", meta.basename);
  h.key("output_block", meta.block_name);
  h.key("file_number", meta.file_number);
  h.key("source_commit", meta.source_commit);
  h.key("mesh_update_seq", meta.mesh_update_seq);
  {
    char hex[24];
    std::snprintf(hex, sizeof(hex), "0x%016llx",
                  static_cast<unsigned long long>(PbinTopologyHash(blocks)));
    h.key("block_topology_hash", hex, "FNV-1a 64 over (level, lx1, lx2, lx3) of the blocks");
  }
  h.section("mesh");
  h.key("ndim", meta.ndim);
  h.key("nx1", meta.nx1); h.key("nx2", meta.nx2); h.key("nx3", meta.nx3);
  h.key("x1min", meta.x1min); h.key("x1max", meta.x1max);
  h.key("x2min", meta.x2min); h.key("x2max", meta.x2max);
  h.key("x3min", meta.x3min); h.key("x3max", meta.x3max);
  h.key("meshblock_nx1", meta.mb_nx1); h.key("meshblock_nx2", meta.mb_nx2);
  h.key("meshblock_nx3", meta.mb_nx3);
  h.key("levels", meta.levels);
  h.key("multilevel", meta.multilevel);
  h.key("adaptive", meta.adaptive);
  {
    const char *faces[6] = {"bc_ix1", "bc_ox1", "bc_ix2", "bc_ox2", "bc_ix3", "bc_ox3"};
    for (int f = 0; f < 6; ++f) h.key(faces[f], meta.bc[f]);
  }
  h.section("particles");
  h.key("zero_mass_rows_excluded", st.zero_mass_rows);
  h.key("invalid_mass_rows", st.invalid_mass_rows);
  h.key("negative_tag_rows", st.negative_tag_rows);
  {
    std::string consts;
    if (plan.constant_sp_ts) consts = "species stopping_time";
    if (plan.constant_mass) consts += consts.empty() ? "mass" : " mass";
    h.key("constant_columns", consts.empty() ? std::string("none") : consts,
          consts.empty() ? nullptr : "values in [constants]");
  }
  h.key("particle_real_precision", meta.single_precision ? "single" : "double");
  h.section("species");
  h.key("nspecies", meta.nspecies);
  h.key("stopping_time_mode", meta.stopping_time_mode);
  if (meta.legacy_species) h.key("dust_to_gas", meta.dust_to_gas);
  h.key("back_reaction", meta.back_reaction);
  for (const auto &l : meta.species_table) h.line(l);
  for (int sp = 0; sp < meta.nspecies; ++sp) {
    std::ostringstream v;
    v << std::setprecision(17) << "input_index " << (sp + 1) << ", tau_s "
      << (sp < static_cast<int>(meta.taus.size()) ? meta.taus[sp]
                                                  : std::numeric_limits<double>::quiet_NaN());
    if (sp < static_cast<int>(meta.species_detail.size())) v << meta.species_detail[sp];
    h.key("species." + std::to_string(sp), v.str());
  }
  h.section("representation");
  for (const auto &l : meta.representation) h.line(l);
  h.section("frame");
  h.key("positions", "lab frame, code length");
  if (meta.shearing_box) {
    h.key("velocity_frame", "shear_relative",
          meta.ndim == 3 ? "v2 relative to -q Omega x1" : "v3 relative to -q Omega x1");
    h.key("shear_q", meta.qshear);
    h.key("shear_omega", meta.omega0);
  } else {
    h.key("velocity_frame", "lab");
  }
  if (meta.compress) {
    h.section("encoding");
    h.key("particle_columns", "shuffle_deflate");
    h.key("chunk_rows", meta.chunk_rows);
    h.key("shuffle", "bytes", "stored[k*rows + i] = raw[i*itemsize + k]");
    h.key("deflate", "zlib", "RFC 1950 stream per chunk, level 1");
    h.key("particle_raw_bytes", raw_bytes);
    h.key("particle_stored_bytes", stored_bytes);
  }
  h.section("columns");
  for (const auto &c : cols) {
    std::ostringstream v;
    v << c.table << " " << c.name << " " << c.dtype << " " << c.count << " " << c.offset << " "
      << c.bytes;
    if (meta.compress) v << (c.encoded ? " shuffle_deflate" : " raw");
    h.key("column", v.str());
  }
  if (meta.compress) {
    h.section("chunks");
    const std::uint64_t nch = NumChunks(ntotal, meta.chunk_rows);
    for (const auto &c : cols) {
      if (!c.encoded) continue;
      std::uint64_t off = c.offset;
      for (std::uint64_t j = 0; j < nch; ++j) {
        const std::uint64_t first = j * meta.chunk_rows;
        const std::uint64_t nrow = (ntotal == 0) ? 0 : std::min(meta.chunk_rows, ntotal - first);
        std::ostringstream v;
        v << c.name << " 0 " << (ntotal == 0 ? 0 : first) << " " << nrow << " " << off << " "
          << c.chunk_bytes[j];
        h.key("chunk", v.str());
        off += c.chunk_bytes[j];
      }
    }
  }
  h.section("constants");
  if (plan.constant_sp_ts) {
    h.key("constant", "particles species " + bo + "u4 0");
    std::ostringstream v;
    v << std::setprecision(17) << "particles stopping_time " << bo << "f8 " << plan.ts0;
    h.key("constant", v.str());
  }
  if (plan.constant_mass) {
    std::ostringstream v;
    v << std::setprecision(17) << "particles mass " << bo << "f8 " << plan.mass;
    h.key("constant", v.str());
  }
  h.section("input");
  h.raw(meta.input_dump);
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
