// Explicit instantiations of the register-resident line-pass and plane
// kernels for line lengths 64, 88.
#include "fastpass.cuh"
#include "pipepass.cuh"
#include "tmapass.cuh"
#include "plane.cuh"

DIS_FAST_INSTANTIATE(8, 8)  // N = 64
DIS_PIPE_INSTANTIATE(8, 8)
template struct pl::PlaneLaunch<8, 8>;
DIS_FAST_INSTANTIATE(8, 11)  // N = 88
DIS_PIPE_INSTANTIATE(8, 11)
DIS_TMA_INSTANTIATE(8, 11)
template struct pl::PlaneLaunch<8, 11>;
