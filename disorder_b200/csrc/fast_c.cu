// Explicit instantiations of the register-resident line-pass and plane
// kernels for line lengths 96, 128.
#include "fastpass.cuh"
#include "pipepass.cuh"
#include "tmapass.cuh"
#include "plane.cuh"

DIS_FAST_INSTANTIATE(8, 12)  // N = 96
DIS_PIPE_INSTANTIATE(8, 12)
DIS_TMA_INSTANTIATE(8, 12)
template struct pl::PlaneLaunch<8, 12>;
DIS_FAST_INSTANTIATE(16, 8)  // N = 128
DIS_PIPE_INSTANTIATE(16, 8)
DIS_TMA_INSTANTIATE(16, 8)
template struct pl::PlaneLaunch<16, 8>;
