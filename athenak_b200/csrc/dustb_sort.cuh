// dustb_sort.cuh -- device CSR (cell -> particles) helpers shared by the sort and the fused
// kernels.
#pragma once
#include <cuda_runtime.h>

namespace dustb {
// scratch bytes of csr_from_keys for ncell cells and n particles
long long csr_scratch_bytes(long long ncell, long long n);
// in-place exclusive scan of n ints (bsum: (n + 4095)/4096 + 1 ints of scratch)
int exclusive_scan(int *a, long long n, int *bsum, cudaStream_t st);
// order/cstart from per-particle keys with explicit scratch (cursor: ncell + 1 ints, bsum:
// scan_bsum_ints(ncell + 1) ints); ordered_runs: order every cell's run by particle index
int csr_build(const int *key, int n, long long ncell, int *cstart, int *order, int *cursor,
              int *bsum, bool ordered_runs, cudaStream_t st);
long long scan_bsum_ints(long long n);
// order/cstart from per-particle keys; cstart[0..ncell) holds the per-cell counts on entry
int csr_from_keys(const int *key, int n, long long ncell, int *cstart, int *order, void *scratch,
                  long long bytes, cudaStream_t st);
}  // namespace dustb
