// Explicit instantiations of the register-resident line-pass kernels
// for line lengths 160, 176.
#include "fastpass.cuh"

DIS_FAST_INSTANTIATE(16, 10)  // N = 160
DIS_FAST_INSTANTIATE(16, 11)  // N = 176
