// dustb_output.cu -- the device side of the particle science file (pbin,
// src/outputs/pbin.cpp): the active rows of the particle arrays in array order (mass != 0,
// ParticleBinaryOutput::LoadOutputData :394-420) with the counts and the mass range the
// header reports (:430-486), one column of those rows packed contiguously
// (PackParticleColumns :322-390), and the byte shuffle of the compressed format (version 3,
// ShuffleDeflate :243-262).  The host writes the file (athenak_b200/host/pbin.cpp).
//
// The compaction is stable: tiles of 2048 rows, read in rounds of 256 consecutive rows
// (coalesced), each row's place from a warp ballot, the warps' counts and the tile's offset;
// the per-tile counts are scanned by one block.  Every result is deterministic.
#include <cfloat>
#include <cstdint>

#include "dustb_common.cuh"

using namespace dustb;

namespace {

constexpr int kT = 256;
constexpr int kRounds = 8;
constexpr int kTile = kT * kRounds;
constexpr int kNStat = 5;      // active, zero, invalid, negative tag, differ

struct Tiles {
  long long *cnt;              // kNStat per tile
  double *mlo, *mhi;           // per tile
  long long *off;              // active-row offset of each tile
};

Tiles tiles_view(void *scratch, long long ntile) {
  char *p = (char *)scratch;
  Tiles t;
  t.cnt = (long long *)p; p += ((ntile * kNStat * 8 + 255) / 256) * 256;
  t.mlo = (double *)p; p += ((ntile * 8 + 255) / 256) * 256;
  t.mhi = (double *)p; p += ((ntile * 8 + 255) / 256) * 256;
  t.off = (long long *)p;
  return t;
}

long long tiles_bytes(long long ntile) {
  return ((ntile * kNStat * 8 + 255) / 256) * 256 + 2 * (((ntile * 8 + 255) / 256) * 256) +
         ((ntile * 8 + 255) / 256) * 256;
}

__device__ __forceinline__ long long warp_sum(long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// the counts and the mass range of one tile (LoadOutputData's checks, the mass range and the
// one-species constant check of WriteOutputFile)
__global__ void k_rows_count(const double *pr, const int *pi, long long stride, int n,
                             double ts0, Tiles T) {
  __shared__ long long s_cnt[kT / 32][kNStat];
  __shared__ double s_lo[kT / 32], s_hi[kT / 32];
  const long long base = (long long)blockIdx.x * kTile;
  long long c[kNStat] = {0, 0, 0, 0, 0};
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (int r = 0; r < kRounds; ++r) {
    const long long p = base + (long long)r * kT + threadIdx.x;
    if (p >= n) break;
    const double m = pr[(long long)DUSTB_IPM * stride + p];
    if (m == 0.0) { ++c[1]; continue; }
    ++c[0];
    if (!(m > 0.0) || !isfinite(m)) ++c[2];
    if (pi[(long long)DUSTB_PTAGH * stride + p] < 0) ++c[3];
    if (pi[(long long)DUSTB_PSP * stride + p] != 0 || pr[(long long)DUSTB_IPTS * stride + p] != ts0)
      ++c[4];
    lo = fmin(lo, m);
    hi = fmax(hi, m);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int q = 0; q < kNStat; ++q) c[q] = warp_sum(c[q]);
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
  }
  if (lane == 0) {
    for (int q = 0; q < kNStat; ++q) s_cnt[w][q] = c[q];
    s_lo[w] = lo; s_hi[w] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t[kNStat] = {0, 0, 0, 0, 0};
    double tl = DBL_MAX, th = -DBL_MAX;
    for (int x = 0; x < kT / 32; ++x) {
      for (int q = 0; q < kNStat; ++q) t[q] += s_cnt[x][q];
      tl = fmin(tl, s_lo[x]); th = fmax(th, s_hi[x]);
    }
    for (int q = 0; q < kNStat; ++q) T.cnt[(long long)blockIdx.x * kNStat + q] = t[q];
    T.mlo[blockIdx.x] = tl; T.mhi[blockIdx.x] = th;
  }
}

// one block: the tiles' exclusive offsets (a carried scan) and the totals
__global__ void k_rows_scan(Tiles T, long long ntile, dustb_pbin_stats *st) {
  __shared__ long long s_w[32];
  __shared__ long long s_tot[kNStat];
  __shared__ double s_lo[32], s_hi[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  long long carry = 0;
  long long tot[kNStat] = {0, 0, 0, 0, 0};
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (long long b0 = 0; b0 < ntile; b0 += blockDim.x) {
    const long long t = b0 + threadIdx.x;
    const long long v = (t < ntile) ? T.cnt[t * kNStat] : 0;
    if (t < ntile) {
      for (int q = 0; q < kNStat; ++q) tot[q] += T.cnt[t * kNStat + q];
      lo = fmin(lo, T.mlo[t]); hi = fmax(hi, T.mhi[t]);
    }
    long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
      long long a = (lane < nw) ? s_w[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, a, o);
        if (lane >= o) a += y;
      }
      s_w[lane] = a;
    }
    __syncthreads();
    const long long before = (w > 0) ? s_w[w - 1] : 0;
    if (t < ntile) T.off[t] = carry + before + x - v;
    carry += s_w[nw - 1];
    __syncthreads();
  }
  // the totals: counts summed (integers, any order), the mass range by fmin / fmax
  for (int q = 0; q < kNStat; ++q) tot[q] = warp_sum(tot[q]);
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_down_sync(0xffffffffu, hi, o));
  }
  if (threadIdx.x < kNStat) s_tot[threadIdx.x] = 0;
  __syncthreads();
  if (lane == 0) {
    for (int q = 0; q < kNStat; ++q) atomicAdd((unsigned long long *)&s_tot[q], (unsigned long long)tot[q]);
    s_lo[w] = lo; s_hi[w] = hi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tl = DBL_MAX, th = -DBL_MAX;
    for (int x = 0; x < nw; ++x) { tl = fmin(tl, s_lo[x]); th = fmax(th, s_hi[x]); }
    st->active_rows = s_tot[0];
    st->zero_mass_rows = s_tot[1];
    st->invalid_mass_rows = s_tot[2];
    st->negative_tag_rows = s_tot[3];
    st->differ_rows = s_tot[4];
    st->mass_min = tl;
    st->mass_max = th;
  }
}

// the active rows of one tile, in array order, at the tile's offset
__global__ void k_rows_write(const double *pr, long long stride, int n, Tiles T, int *idx) {
  __shared__ int s_w[kT / 32];
  const long long base = (long long)blockIdx.x * kTile;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  long long at = T.off[blockIdx.x];
  for (int r = 0; r < kRounds; ++r) {
    const long long p = base + (long long)r * kT + threadIdx.x;
    const bool act = p < n && pr[(long long)DUSTB_IPM * stride + p] != 0.0;
    const unsigned b = __ballot_sync(0xffffffffu, act);
    if (lane == 0) s_w[w] = __popc(b);
    __syncthreads();
    int before = 0, total = 0;
    for (int x = 0; x < kT / 32; ++x) {
      if (x < w) before += s_w[x];
      total += s_w[x];
    }
    if (act) idx[at + before + __popc(b & ((1u << lane) - 1u))] = (int)p;
    at += total;
    __syncthreads();
  }
}

__global__ void k_pack(const double *pr, const int *pi, long long stride, const int *idx, int n,
                       int column, int single, void *out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const long long p = idx[q];
    if (column == DUSTB_PBIN_ID) {
      const unsigned lo = (unsigned)pi[(long long)DUSTB_PTAG * stride + p];
      const unsigned hi = (unsigned)pi[(long long)DUSTB_PTAGH * stride + p];
      ((unsigned long long *)out)[q] = ((unsigned long long)hi << 32) | lo;
    } else if (column == DUSTB_PBIN_SPECIES) {
      ((unsigned *)out)[q] = (unsigned)pi[(long long)DUSTB_PSP * stride + p];
    } else {
      int row = DUSTB_IPX;
      switch (column) {
        case DUSTB_PBIN_X2: row = DUSTB_IPY; break;
        case DUSTB_PBIN_X3: row = DUSTB_IPZ; break;
        case DUSTB_PBIN_V1: row = DUSTB_IPVX; break;
        case DUSTB_PBIN_V2: row = DUSTB_IPVY; break;
        case DUSTB_PBIN_V3: row = DUSTB_IPVZ; break;
        case DUSTB_PBIN_MASS: row = DUSTB_IPM; break;
        case DUSTB_PBIN_STOPPING_TIME: row = DUSTB_IPTS; break;
        default: break;
      }
      const double v = pr[(long long)row * stride + p];
      if (single) ((float *)out)[q] = (float)v;
      else ((double *)out)[q] = v;
    }
  }
}

// stored[k * rows + i] = raw[i * itemsize + k] within each chunk of chunk_rows rows
__global__ void k_shuffle(const unsigned char *in, long long n, int size, long long chunk_rows,
                          unsigned char *out) {
  const long long total = n * size, per = chunk_rows * size;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const long long j = o / per;
    const long long r0 = j * chunk_rows;
    const long long rows = (n - r0 < chunk_rows) ? n - r0 : chunk_rows;
    const long long local = o - j * per;
    const long long k = local / rows, i = local - k * rows;
    out[o] = in[(r0 + i) * size + k];
  }
}

inline unsigned grid_for(long long n) {
  long long b = (n + kT - 1) / kT;
  if (b > 148LL * 16) b = 148LL * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

}  // namespace

extern "C" {

long long dustb_pbin_scratch_bytes(int npart) {
  if (npart < 0) return -1;
  const long long ntile = ((long long)npart + kTile - 1) / kTile;
  return tiles_bytes(ntile > 0 ? ntile : 1);
}

int dustb_pbin_rows(const dustb_ctx *c, int *idx, dustb_pbin_stats *stats, double ts0,
                    void *scratch, long long scratch_bytes, void *stream) {
  if (!c || !stats || !scratch) return DUSTB_EINVAL;
  const int n = c->part.npart;
  if (n < 0 || (n > 0 && (!idx || !c->part.pr || !c->part.pi)) || n > c->part.stride)
    return DUSTB_EINVAL;
  if (scratch_bytes < dustb_pbin_scratch_bytes(n)) return DUSTB_ESCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  const long long ntile = ((long long)n + kTile - 1) / kTile;
  const Tiles T = tiles_view(scratch, ntile > 0 ? ntile : 1);
  if (ntile > 0)
    k_rows_count<<<(unsigned)ntile, kT, 0, st>>>(c->part.pr, c->part.pi, c->part.stride, n, ts0, T);
  k_rows_scan<<<1, 1024, 0, st>>>(T, ntile, stats);
  if (ntile > 0)
    k_rows_write<<<(unsigned)ntile, kT, 0, st>>>(c->part.pr, c->part.stride, n, T, idx);
  return dustb_host::launch_status("pbin_rows");
}

int dustb_pbin_pack(const dustb_ctx *c, const int *idx, int n, int column, int single, void *out,
                    void *stream) {
  if (!c || n < 0 || (n > 0 && (!idx || !out))) return DUSTB_EINVAL;
  if (column < DUSTB_PBIN_ID || column > DUSTB_PBIN_STOPPING_TIME) return DUSTB_EINVAL;
  if (n > 0)
    k_pack<<<grid_for(n), kT, 0, (cudaStream_t)stream>>>(c->part.pr, c->part.pi, c->part.stride,
                                                         idx, n, column, single, out);
  return dustb_host::launch_status("pbin_pack");
}

int dustb_pbin_shuffle(const void *in, long long rows, int itemsize, long long chunk_rows,
                       void *out, void *stream) {
  if (rows < 0 || itemsize <= 0 || chunk_rows <= 0 || (rows > 0 && (!in || !out)))
    return DUSTB_EINVAL;
  if (rows > 0)
    k_shuffle<<<grid_for(rows * itemsize), kT, 0, (cudaStream_t)stream>>>(
        (const unsigned char *)in, rows, itemsize, chunk_rows, (unsigned char *)out);
  return dustb_host::launch_status("pbin_shuffle");
}

}  // extern "C"
