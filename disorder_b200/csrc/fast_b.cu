// Explicit instantiations of the register-resident line-pass kernels
// for line lengths 64, 88.
#include "fastpass.cuh"

DIS_FAST_INSTANTIATE(8, 8)  // N = 64
DIS_FAST_INSTANTIATE(8, 11)  // N = 88
