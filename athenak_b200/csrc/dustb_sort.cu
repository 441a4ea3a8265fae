// dustb_sort.cu -- particle cell index (a CSR over cells) and the cell sort of the
// particle SoA (DustGasDrag::SortParticles, src/dust/dust_cloud_device.cpp:1881-1977).
//
// The reference sorts 64-bit keys (block*ncell + cell)*npart + p with thrust::sort.  The same
// permutation comes from a counting sort over the cell key (one bucket per cell: the bucket
// count fits the mesh arrays anyway), followed by ordering each bucket by particle index.
// Steps: key + histogram (atomics on the cell counters), exclusive scan of the counters,
// scatter of the particle indices with per-cell cursors, per-cell sort of the (short)
// index runs.  Every result is deterministic.
#include <atomic>
#include <cstdint>
#include <cstdio>

#include "dustb_common.cuh"
#include "dustb_sort.cuh"

using namespace dustb;

namespace {

constexpr int kT = 256;
constexpr int kScanT = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanT * kScanItems;

inline unsigned nblk(long long n, int t = kT) {
  long long b = (n + t - 1) / t;
  return (unsigned)(b < 1 ? 1 : b);
}

// SortParticles' key of particle p (dust_cloud_device.cpp:1900-1916)
__global__ void k_keys(const double *pr, const int *pi, long long stride, int npart,
                       const double *mb, int gids, int nmb, int nx1, int nx2, int nx3, int z3,
                       int *key, int *count) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npart) return;
  int m = pi[(long long)DUSTB_PGID * stride + p] - gids;
  m = (m < 0) ? 0 : ((m >= nmb) ? nmb - 1 : m);
  const double *s = mb + (long long)m * 9;
  int i = (int)floor((pr[(long long)DUSTB_IPX * stride + p] - s[X1MIN]) / s[DX1]);
  int j = (int)floor((pr[(long long)DUSTB_IPY * stride + p] - s[X2MIN]) / s[DX2]);
  i = (i < 0) ? 0 : ((i >= nx1) ? nx1 - 1 : i);
  j = (j < 0) ? 0 : ((j >= nx2) ? nx2 - 1 : j);
  int k = 0;
  if (z3) {
    k = (int)floor((pr[(long long)DUSTB_IPZ * stride + p] - s[X3MIN]) / s[DX3]);
    k = (k < 0) ? 0 : ((k >= nx3) ? nx3 - 1 : k);
  }
  const int c = m * (nx1 * nx2 * nx3) + (k * nx2 + j) * nx1 + i;
  key[p] = c;
  atomicAdd(&count[c], 1);
}

// ---- exclusive scan of n ints in place (three kernels) ---------------------------------
__device__ __forceinline__ int block_excl_scan(int v, int *sh, int &total) {
  // warp inclusive scan
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sh[lane] = w;    // inclusive warp totals
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  int base = (warp > 0) ? sh[warp - 1] : 0;
  __syncthreads();
  return base + x - v;
}

__global__ void k_scan_reduce(const int *a, long long n, int *bsum) {
  __shared__ int sh[32];
  long long base = (long long)blockIdx.x * kScanTile;
  int s = 0;
  for (int r = 0; r < kScanItems; ++r) {
    long long idx = base + (long long)r * kScanT + threadIdx.x;
    if (idx < n) s += a[idx];
  }
  int total;
  block_excl_scan(s, sh, total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// one block: exclusive scan of nb block sums, chunk after chunk with a carry
__global__ void k_scan_sums(int *bsum, int nb) {
  __shared__ int sh[32];
  int carry = 0;
  for (int base = 0; base < nb; base += kScanT) {
    int idx = base + threadIdx.x;
    int v = (idx < nb) ? bsum[idx] : 0;
    int total;
    int ex = block_excl_scan(v, sh, total);
    if (idx < nb) bsum[idx] = carry + ex;
    carry += total;
    __syncthreads();
  }
}

__global__ void k_scan_apply(int *a, long long n, const int *bsum) {
  __shared__ int sh[32];
  long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
  for (int r = 0; r < kScanItems; ++r) {
    long long idx = base + r;
    v[r] = (idx < n) ? a[idx] : 0;
    s += v[r];
  }
  int total;
  int ex = block_excl_scan(s, sh, total) + bsum[blockIdx.x];
  for (int r = 0; r < kScanItems; ++r) {
    long long idx = base + r;
    if (idx < n) a[idx] = ex;
    ex += v[r];
  }
}

// lanes of a warp with the same key take consecutive slots from one atomic (keys of
// nearly cell-sorted particles come in runs)
__global__ void k_fill(const int *key, int npart, int *cursor, int *order) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = p < npart;
  const unsigned act = __ballot_sync(0xffffffffu, live);
  if (!live) return;
  const int k = key[p];
  const unsigned peers = __match_any_sync(act, k);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  const int rank = __popc(peers & ((1u << lane) - 1u));
  int base = 0;
  if (lane == leader) base = atomicAdd(&cursor[k], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  order[base + rank] = p;
}

// order every cell's run by particle index: insertion sort for short runs, heap sort
// for long ones (both in place, deterministic)
__device__ void sift_down(int *a, int root, int n) {
  while (true) {
    int child = 2 * root + 1;
    if (child >= n) return;
    if (child + 1 < n && a[child] < a[child + 1]) ++child;
    if (a[root] >= a[child]) return;
    int t = a[root]; a[root] = a[child]; a[child] = t;
    root = child;
  }
}

__global__ void k_sort_runs(const int *cstart, long long ncell, int *order) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int b = cstart[c], e = cstart[c + 1];
  int n = e - b;
  if (n < 2) return;
  int *a = order + b;
  if (n <= 48) {
    for (int x = 1; x < n; ++x) {
      int v = a[x];
      int y = x - 1;
      while (y >= 0 && a[y] > v) { a[y + 1] = a[y]; --y; }
      a[y + 1] = v;
    }
    return;
  }
  for (int r = n / 2 - 1; r >= 0; --r) sift_down(a, r, n);
  for (int x = n - 1; x > 0; --x) {
    int t = a[0]; a[0] = a[x]; a[x] = t;
    sift_down(a, 0, x);
  }
}

// every row of particle order[k] into slot k of the spare arrays
__global__ void k_move(const double *pr, const int *pi, long long stride, int npart,
                       const int *order, double *npr, int *npi) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npart) return;
  int p = order[k];
  for (int r = 0; r < DUSTB_NREAL; ++r) npr[(long long)r * stride + k] = pr[(long long)r * stride + p];
  for (int r = 0; r < DUSTB_NINT; ++r) npi[(long long)r * stride + k] = pi[(long long)r * stride + p];
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

namespace dustb {

long long csr_scratch_bytes(long long ncell, long long n) {
  long long nb = (ncell + 1 + kScanTile - 1) / kScanTile;
  return (long long)(align256(sizeof(int) * (size_t)(n > 0 ? n : 1)) +
                     align256(sizeof(int) * (size_t)(ncell + 1)) +
                     align256(sizeof(int) * (size_t)(nb + 1)));
}

int exclusive_scan(int *a, long long n, int *bsum, cudaStream_t st) {
  long long nb = (n + kScanTile - 1) / kScanTile;
  k_scan_reduce<<<(unsigned)nb, kScanT, 0, st>>>(a, n, bsum);
  k_scan_sums<<<1, kScanT, 0, st>>>(bsum, (int)nb);
  k_scan_apply<<<(unsigned)nb, kScanT, 0, st>>>(a, n, bsum);
  return dustb_host::launch_status("exclusive_scan");
}

// CSR from precomputed keys: key[n] in [0, ncell); cstart (ncell + 1 ints) holds the
// per-cell counts on entry; cursor (ncell + 1 ints) and bsum are scratch.
int csr_build(const int *key, int n, long long ncell, int *cstart, int *order, int *cursor,
              int *bsum, bool ordered_runs, cudaStream_t st) {
  int rc = exclusive_scan(cstart, ncell + 1, bsum, st);
  if (rc) return rc;
  cudaMemcpyAsync(cursor, cstart, sizeof(int) * (size_t)(ncell + 1), cudaMemcpyDeviceToDevice, st);
  if (n > 0) k_fill<<<nblk(n), kT, 0, st>>>(key, n, cursor, order);
  if (ordered_runs) k_sort_runs<<<nblk(ncell), kT, 0, st>>>(cstart, ncell, order);
  return dustb_host::launch_status("csr_build");
}

long long scan_bsum_ints(long long n) { return (n + kScanTile - 1) / kScanTile + 1; }

int csr_from_keys(const int *key, int n, long long ncell, int *cstart, int *order, void *scratch,
                  long long bytes, cudaStream_t st) {
  if (bytes < csr_scratch_bytes(ncell, n)) return DUSTB_ESCRATCH;
  char *p = (char *)scratch;
  p += align256(sizeof(int) * (size_t)(n > 0 ? n : 1));   // key slot (dustb_cell_index)
  int *cursor = (int *)p; p += align256(sizeof(int) * (size_t)(ncell + 1));
  int *bsum = (int *)p;
  return csr_build(key, n, ncell, cstart, order, cursor, bsum, true, st);
}

}  // namespace dustb

extern "C" {

long long dustb_sort_scratch_bytes(const dustb_mesh *mesh, int npart) {
  if (!mesh) return -1;
  long long ncell = (long long)mesh->nmb * mesh->nx1 * (mesh->multi_d ? mesh->nx2 : 1) *
                    (mesh->three_d ? mesh->nx3 : 1);
  // keys + CSR scratch, then order + cstart of dustb_sort_by_cell
  return csr_scratch_bytes(ncell, npart) +
         (long long)(align256(sizeof(int) * (size_t)(npart > 0 ? npart : 1)) +
                     align256(sizeof(int) * (size_t)(ncell + 1)));
}

int dustb_cell_index(const dustb_ctx *c, int *order, int *cstart, void *scratch,
                     long long scratch_bytes, void *stream) {
  if (!c || !order || !cstart || !scratch) return DUSTB_EINVAL;
  const dustb_mesh &ms = c->mesh;
  const int nx2 = ms.multi_d ? ms.nx2 : 1, nx3 = ms.three_d ? ms.nx3 : 1;
  const long long ncell = (long long)ms.nmb * ms.nx1 * nx2 * nx3;
  if (ncell >= (1LL << 31)) return DUSTB_EUNSUP;
  const int n = c->part.npart;
  if (scratch_bytes < csr_scratch_bytes(ncell, n)) return DUSTB_ESCRATCH;
  cudaStream_t st = (cudaStream_t)stream;
  int *key = (int *)scratch;
  cudaMemsetAsync(cstart, 0, sizeof(int) * (size_t)(ncell + 1), st);
  if (n > 0)
    k_keys<<<nblk(n), kT, 0, st>>>(c->part.pr, c->part.pi, c->part.stride, n, ms.mb_size, ms.gids,
                                   ms.nmb, ms.nx1, nx2, nx3, ms.three_d, key, cstart);
  return csr_from_keys(key, n, ncell, cstart, order, scratch, scratch_bytes, st);
}

int dustb_sort_by_cell(const dustb_ctx *c, double *spare_pr, int *spare_pi, void *scratch,
                       long long scratch_bytes, void *stream) {
  if (!c || !spare_pr || !spare_pi || !scratch) return DUSTB_EINVAL;
  const dustb_mesh &ms = c->mesh;
  const int n = c->part.npart;
  if (scratch_bytes < dustb_sort_scratch_bytes(&ms, n)) return DUSTB_ESCRATCH;
  const long long ncell = (long long)ms.nmb * ms.nx1 * (ms.multi_d ? ms.nx2 : 1) *
                          (ms.three_d ? ms.nx3 : 1);
  const long long base = csr_scratch_bytes(ncell, n);
  int *order = (int *)((char *)scratch + base);
  int *cstart = (int *)((char *)scratch + base + align256(sizeof(int) * (size_t)(n > 0 ? n : 1)));
  int rc = dustb_cell_index(c, order, cstart, scratch, base, stream);
  if (rc) return rc;
  if (n > 0)
    k_move<<<nblk(n), kT, 0, (cudaStream_t)stream>>>(c->part.pr, c->part.pi, c->part.stride, n,
                                                       order, spare_pr, spare_pi);
  return dustb_host::launch_status("sort_by_cell");
}

}  // extern "C"

// ---- the cloud order index (DustGasDrag::UpdateCloudOrder) -------------------------------
namespace {

// the 64-bit tag of particle p: PTAG the low word, PTAGH the high (two's complement words)
__device__ __forceinline__ unsigned long long tag_of(const int *pi, long long stride, int p) {
  const unsigned lo = (unsigned)pi[(long long)DUSTB_PTAG * stride + p];
  const unsigned hi = (unsigned)pi[(long long)DUSTB_PTAGH * stride + p];
  return ((unsigned long long)hi << 32) | (unsigned long long)lo;
}

// the tag of the particle each slot k indexes: ord given (the key order), or written as the
// identity (identity = 1: after a sort in cell order)
__global__ void k_order_tags(const int *pi, long long stride, int n, int *ord, int identity,
                             unsigned long long *tag) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int p = k;
  if (identity) ord[k] = k;
  else p = ord[k];
  tag[k] = tag_of(pi, stride, p);
}

// entries k < n whose slot is out of range or holds another particle than when indexed
__global__ void k_order_check(const int *pi, long long stride, int npart, const int *ord,
                              const unsigned long long *tag, int n, int *bad) {
  int cnt = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int p = ord[k];
    if (p < 0 || p >= npart || tag_of(pi, stride, p) != tag[k]) ++cnt;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(bad, cnt);
}

}  // namespace

extern "C" {

int dustb_cloud_order(const dustb_ctx *c, int *ord, unsigned long long *tag, void *scratch,
                      long long scratch_bytes, void *stream) {
  if (!c || !ord || !tag || !scratch) return DUSTB_EINVAL;
  const dustb_mesh &ms = c->mesh;
  const int n = c->part.npart;
  if (scratch_bytes < dustb_sort_scratch_bytes(&ms, n)) return DUSTB_ESCRATCH;
  const long long ncell = (long long)ms.nmb * ms.nx1 * (ms.multi_d ? ms.nx2 : 1) *
                          (ms.three_d ? ms.nx3 : 1);
  const long long base = csr_scratch_bytes(ncell, n);
  // the per-cell starts are not returned: they sit behind the key scratch
  int *cstart = (int *)((char *)scratch + base);
  int rc = dustb_cell_index(c, ord, cstart, scratch, base, stream);
  if (rc) return rc;
  if (n > 0)
    k_order_tags<<<nblk(n), kT, 0, (cudaStream_t)stream>>>(c->part.pi, c->part.stride, n, ord, 0,
                                                             tag);
  return dustb_host::launch_status("cloud_order");
}

int dustb_cloud_order_identity(const dustb_ctx *c, int *ord, unsigned long long *tag,
                               void *stream) {
  if (!c || !ord || !tag) return DUSTB_EINVAL;
  const int n = c->part.npart;
  if (n > 0)
    k_order_tags<<<nblk(n), kT, 0, (cudaStream_t)stream>>>(c->part.pi, c->part.stride, n, ord, 1,
                                                             tag);
  return dustb_host::launch_status("cloud_order_identity");
}

int dustb_cloud_order_check(const dustb_ctx *c, const int *ord, const unsigned long long *tag,
                            int n, int *bad, void *stream) {
  if (!c || !bad || n < 0 || (n > 0 && (!ord || !tag))) return DUSTB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(bad, 0, sizeof(int), st);
  if (n > 0) {
    const unsigned g = nblk(n) < 148u * 8u ? nblk(n) : 148u * 8u;
    k_order_check<<<g, kT, 0, st>>>(c->part.pi, c->part.stride, c->part.npart, ord, tag, n, bad);
  }
  return dustb_host::launch_status("cloud_order_check");
}

}  // extern "C"

// ---- cell index without any allocation ---------------------------------------------------
// For host codes that cannot allocate device memory at the point of the call (a code whose
// device memory all comes from its own pool reserved at start-up, or one that must not make
// the synchronising cudaMalloc/cudaFree calls inside its time step): the scratch of the cell
// index lives in this file-scope device array instead of a caller buffer.  Every GPU that
// loads the library holds it until the process exits.
static __device__ __align__(256) unsigned char g_cell_index_scratch[DUSTB_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
// the array's device address on each device.  The name g_cell_index_scratch in host code is
// only a host-side handle, so the address is asked from the runtime, once per device, with
// that device current.  Atomic slots: host threads making their first call on one device at
// the same time may both look the address up (the same value) and store it without a race.
// A cudaDeviceReset unloads the module, so the cached address is stale after it:
// dustb_cell_index_static_reset() clears the slots for such a caller.
std::atomic<void *> g_cell_index_scratch_ptr[kMaxDevices];
}  // namespace

extern "C" int dustb_cell_index_static(const dustb_ctx *c, int *order, int *cstart,
                                       void *stream) {
  if (!c || !order || !cstart) return DUSTB_EINVAL;
  const dustb_mesh &ms = c->mesh;
  const long long ncell = (long long)ms.nmb * ms.nx1 * (ms.multi_d ? ms.nx2 : 1) *
                          (ms.three_d ? ms.nx3 : 1);
  if (ncell >= (1LL << 31)) return DUSTB_EUNSUP;
  const long long need = csr_scratch_bytes(ncell, c->part.npart);
  if (need > (long long)DUSTB_STATIC_SCRATCH_BYTES) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "dustb_cell_index_static: %lld particles and %lld cells need %lld scratch bytes, "
             "more than the fixed %lld",
             (long long)c->part.npart, ncell, need, (long long)DUSTB_STATIC_SCRATCH_BYTES);
    dustb_host::set_message(msg);
    return DUSTB_ESCRATCH;
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { dustb_host::set_error("dustb_cell_index_static: cudaGetDevice", e); return DUSTB_ELAUNCH; }
  if (dev < 0 || dev >= kMaxDevices) {
    char msg[128];
    snprintf(msg, sizeof(msg), "dustb_cell_index_static: device ordinal %d is not below the %d "
             "devices the address cache holds", dev, kMaxDevices);
    dustb_host::set_message(msg);
    return DUSTB_EUNSUP;
  }
  void *ptr = g_cell_index_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!ptr) {
    e = cudaGetSymbolAddress(&ptr, g_cell_index_scratch);
    if (e != cudaSuccess || !ptr) {
      dustb_host::set_error("dustb_cell_index_static: cudaGetSymbolAddress", e);
      return DUSTB_ELAUNCH;
    }
    g_cell_index_scratch_ptr[dev].store(ptr, std::memory_order_release);
  }
  // nothing in the array needs to start at zero: the keys, the cursors and the scan sums are
  // all written before they are read, and the per-cell counts are kept in the caller's
  // cstart, which dustb_cell_index clears
  return dustb_cell_index(c, order, cstart, ptr, (long long)DUSTB_STATIC_SCRATCH_BYTES, stream);
}

extern "C" int dustb_cell_index_static_reset(void) {
  for (int d = 0; d < kMaxDevices; ++d) g_cell_index_scratch_ptr[d].store(nullptr);
  return DUSTB_OK;
}
