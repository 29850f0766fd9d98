// Explicit instantiations of the register-resident line-pass and plane
// kernels for line lengths 160, 176.
#include "fastpass.cuh"
#include "pipepass.cuh"
#include "tmapass.cuh"
#include "plane.cuh"

DIS_FAST_INSTANTIATE(16, 10)  // N = 160
DIS_PIPE_INSTANTIATE(16, 10)
DIS_TMA_INSTANTIATE(16, 10)
template struct pl::PlaneLaunch<16, 10>;
DIS_FAST_INSTANTIATE(16, 11)  // N = 176
DIS_PIPE_INSTANTIATE(16, 11)
DIS_TMA_INSTANTIATE(16, 11)
template struct pl::PlaneLaunch<16, 11>;
