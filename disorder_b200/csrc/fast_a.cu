// Explicit instantiations of the register-resident line-pass kernels
// for line lengths 16, 32, 44.
#include "fastpass.cuh"

DIS_FAST_INSTANTIATE(4, 4)  // N = 16
DIS_FAST_INSTANTIATE(8, 4)  // N = 32
DIS_FAST_INSTANTIATE(4, 11)  // N = 44
