// Host-side entry points of the register-resident line-pass kernels.
#pragma once
#include "internal.h"

// Factorisation used for a line length n (0 when n has no fast kernel).
bool dis_fast_factor(int n, int* F1, int* F2);
// Each returns false when n has no fast kernel (the caller then uses the
// generic shared-memory Stockham kernels).
bool dis_fast_line(const LinePassArgs& a, const float2* tw, cudaStream_t s);
bool dis_fast_expand(int n, const CoilArgs& a, const float2* z, float2* A, const float2* tw, cudaStream_t s);
bool dis_fast_combine(int n, const CoilArgs& a, const float2* A, float2* u, float scale, const float2* tw,
                      cudaStream_t s);
bool dis_fast_axis1(int n, int mode, const CoilArgs& a, float2* A, float2* y, const float2* ymeas, long long ld,
                    int n3off, int N3y, float scale, const float* wmap, const float* We, const float* Mb,
                    const disorder_plan_s* plan, const float2* tw, cudaStream_t s);
