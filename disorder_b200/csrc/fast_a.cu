// Explicit instantiations of the register-resident line-pass and plane
// kernels for line lengths 16, 32, 44.
#include "fastpass.cuh"
#include "pipepass.cuh"
#include "tmapass.cuh"
#include "plane.cuh"

DIS_FAST_INSTANTIATE(4, 4)  // N = 16
DIS_PIPE_INSTANTIATE(4, 4)
template struct pl::PlaneLaunch<4, 4>;
DIS_FAST_INSTANTIATE(8, 4)  // N = 32
DIS_PIPE_INSTANTIATE(8, 4)
template struct pl::PlaneLaunch<8, 4>;
DIS_FAST_INSTANTIATE(4, 11)  // N = 44
DIS_PIPE_INSTANTIATE(4, 11)
DIS_TMA_INSTANTIATE(4, 11)
template struct pl::PlaneLaunch<4, 11>;
