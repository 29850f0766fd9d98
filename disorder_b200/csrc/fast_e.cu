// Explicit instantiations of the register-resident line-pass kernels
// for line lengths 192, 256.
#include "fastpass.cuh"

DIS_FAST_INSTANTIATE(16, 12)  // N = 192
DIS_FAST_INSTANTIATE(16, 16)  // N = 256
