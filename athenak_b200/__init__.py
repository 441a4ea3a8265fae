"""B200-native dust particle-drag step (gather + kick + deposit) behind a C ABI.

The CUDA kernels live in csrc/ and build into libdustb.so (build.py); include/dustb.h is the
ABI.  drag.DeviceDust (FP64, reference layout) and mixed.MixedDust (mixed precision) are
the host front ends used by the tests and the benchmark.
"""
