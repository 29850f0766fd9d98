// Explicit instantiations of the register-resident line-pass and plane
// kernels for line lengths 192, 256.
#include "fastpass.cuh"
#include "pipepass.cuh"
#include "tmapass.cuh"
#include "plane.cuh"

DIS_FAST_INSTANTIATE(16, 12)  // N = 192
DIS_PIPE_INSTANTIATE(16, 12)
DIS_TMA_INSTANTIATE(16, 12)
template struct pl::PlaneLaunch<16, 12>;
DIS_FAST_INSTANTIATE(16, 16)  // N = 256
DIS_PIPE_INSTANTIATE(16, 16)
DIS_TMA_INSTANTIATE(16, 16)
template struct pl::PlaneLaunch<16, 16>;
