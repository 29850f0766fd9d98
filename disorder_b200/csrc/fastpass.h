// Host-side entry points of the register-resident line-pass kernels.
#pragma once
#include "internal.h"

// Factorisation used for a line length n (0 when n has no fast kernel).
bool dis_fast_factor(int n, int* F1, int* F2);
// Each returns false when n has no fast kernel (the caller then uses the
// generic shared-memory Stockham kernels).
bool dis_fast_line(const LinePassArgs& a, const float2* tw, cudaStream_t s);
// Pipelined persistent kernel (pipepass.cuh) for the single-input passes;
// false when the pass does not fit it.
bool dis_fast_pipe(const LinePassArgs& a, const float2* tw, cudaStream_t s);
// Pipelined weighted dim-2 pass of the normal operator (pipepass.cuh,
// wpipe_kernel) for line length n = N2; false when it does not apply.
bool dis_fast_wpipe(int n, const CoilArgs& a, float2* A, const float* wmap, const float2* tw, cudaStream_t s);
// TMA tile-copy variants (tmapass.cuh) of the strided transform passes and
// of the weighted pass; false when the pass does not fit them.
bool dis_fast_tma_line(disorder_ctx_s* ctx, const LinePassArgs& a);
// With ys non-null the weighted pass also writes the forward samples (encode's
// layout and scale) into ys.
bool dis_fast_tma_weight(disorder_ctx_s* ctx, const CoilArgs& a, float2* A, const float* wmap, const float2* tw,
                         const disorder_plan_s* plan = nullptr, float2* ys = nullptr, long long ld = 0, int n3off = 0,
                         int N3y = 0, float scale = 1.f);
bool dis_fast_tma_gather(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* A,
                         float2* y, long long y_ld, int y_n3off, int y_N3, const float2* y_meas, float scale);
bool dis_fast_tma_scatter(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* y,
                          long long y_ld, int y_n3off, int y_N3, const float* We, const float* Mb, float2* A);
bool dis_fast_expand(int n, const CoilArgs& a, const float2* z, float2* A, const float2* tw, cudaStream_t s);
bool dis_fast_combine(int n, const CoilArgs& a, const float2* A, float2* u, float scale, const float2* tw,
                      cudaStream_t s);
bool dis_fast_axis1(int n, int mode, const CoilArgs& a, float2* A, float2* y, const float2* ymeas, long long ld,
                    int n3off, int N3y, float scale, const float* wmap, const float* We, const float* Mb,
                    const disorder_plan_s* plan, const float2* tw, cudaStream_t s);

namespace pl {
struct PlaneArgs;
}
// Fused coil stage (plane.cuh). mode: 0 encode, 1 decode, 2 encodedecode.
// Returns false when N1 has no fast kernel or the shared memory does not fit.
bool dis_fast_plane(int n1, int mode, const pl::PlaneArgs& a, const float2* tw1, const float2* tw2, int n_slots,
                    cudaStream_t s);
size_t dis_plane_smem(int n1, int N2, int C, int max_ns);
