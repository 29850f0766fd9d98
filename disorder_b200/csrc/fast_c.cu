// Explicit instantiations of the register-resident line-pass kernels
// for line lengths 96, 128.
#include "fastpass.cuh"

DIS_FAST_INSTANTIATE(8, 12)  // N = 96
DIS_FAST_INSTANTIATE(16, 8)  // N = 128
