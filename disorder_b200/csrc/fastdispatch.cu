// Size dispatch of the register-resident line-pass kernels. The kernels are
// instantiated in fast_[a-e].cu (one translation unit per group of sizes).
#include "fastpass.cuh"
#include "fastpass.h"
#include "pipepass.cuh"
#include "plane.cuh"

#define DIS_EXTERN_PIPE(F1, F2)                 \
  extern template struct fp::PipeLaunch<F1, F2>; \
  extern template struct fp::WPipeLaunch<F1, F2>;
DIS_EXTERN_PIPE(4, 4)
DIS_EXTERN_PIPE(8, 4)
DIS_EXTERN_PIPE(4, 11)
DIS_EXTERN_PIPE(8, 8)
DIS_EXTERN_PIPE(8, 11)
DIS_EXTERN_PIPE(8, 12)
DIS_EXTERN_PIPE(16, 8)
DIS_EXTERN_PIPE(16, 10)
DIS_EXTERN_PIPE(16, 11)
DIS_EXTERN_PIPE(16, 12)
DIS_EXTERN_PIPE(16, 16)
#undef DIS_EXTERN_PIPE

extern template struct fp::Launch<4, 4>;
extern template struct fp::Launch<8, 4>;
extern template struct fp::Launch<4, 11>;
extern template struct fp::Launch<8, 8>;
extern template struct fp::Launch<8, 11>;
extern template struct fp::Launch<8, 12>;
extern template struct fp::Launch<16, 8>;
extern template struct fp::Launch<16, 10>;
extern template struct fp::Launch<16, 11>;
extern template struct fp::Launch<16, 12>;
extern template struct fp::Launch<16, 16>;

extern template struct pl::PlaneLaunch<4, 4>;
extern template struct pl::PlaneLaunch<8, 4>;
extern template struct pl::PlaneLaunch<4, 11>;
extern template struct pl::PlaneLaunch<8, 8>;
extern template struct pl::PlaneLaunch<8, 11>;
extern template struct pl::PlaneLaunch<8, 12>;
extern template struct pl::PlaneLaunch<16, 8>;
extern template struct pl::PlaneLaunch<16, 10>;
extern template struct pl::PlaneLaunch<16, 11>;
extern template struct pl::PlaneLaunch<16, 12>;
extern template struct pl::PlaneLaunch<16, 16>;

bool dis_fast_factor(int n, int* F1, int* F2) {
  switch (n) {
    case 16: *F1 = 4; *F2 = 4; return true;
    case 32: *F1 = 8; *F2 = 4; return true;
    case 44: *F1 = 4; *F2 = 11; return true;
    case 64: *F1 = 8; *F2 = 8; return true;
    case 88: *F1 = 8; *F2 = 11; return true;
    case 96: *F1 = 8; *F2 = 12; return true;
    case 128: *F1 = 16; *F2 = 8; return true;
    case 160: *F1 = 16; *F2 = 10; return true;
    case 176: *F1 = 16; *F2 = 11; return true;
    case 192: *F1 = 16; *F2 = 12; return true;
    case 256: *F1 = 16; *F2 = 16; return true;
    default: return false;
  }
}

bool dis_fast_pipe(const LinePassArgs& a, const float2* tw, cudaStream_t s) {
  switch (a.N[a.axis]) {
    case 16: return fp::PipeLaunch<4, 4>::run(a, tw, s);
    case 32: return fp::PipeLaunch<8, 4>::run(a, tw, s);
    case 44: return fp::PipeLaunch<4, 11>::run(a, tw, s);
    case 64: return fp::PipeLaunch<8, 8>::run(a, tw, s);
    case 88: return fp::PipeLaunch<8, 11>::run(a, tw, s);
    case 96: return fp::PipeLaunch<8, 12>::run(a, tw, s);
    case 128: return fp::PipeLaunch<16, 8>::run(a, tw, s);
    case 160: return fp::PipeLaunch<16, 10>::run(a, tw, s);
    case 176: return fp::PipeLaunch<16, 11>::run(a, tw, s);
    case 192: return fp::PipeLaunch<16, 12>::run(a, tw, s);
    case 256: return fp::PipeLaunch<16, 16>::run(a, tw, s);
    default: return false;
  }
}

bool dis_fast_wpipe(int n, const CoilArgs& a, float2* A, const float* wmap, const float2* tw, cudaStream_t s) {
  switch (n) {
    case 16: return fp::WPipeLaunch<4, 4>::run(a, A, wmap, tw, s);
    case 32: return fp::WPipeLaunch<8, 4>::run(a, A, wmap, tw, s);
    case 44: return fp::WPipeLaunch<4, 11>::run(a, A, wmap, tw, s);
    case 64: return fp::WPipeLaunch<8, 8>::run(a, A, wmap, tw, s);
    case 88: return fp::WPipeLaunch<8, 11>::run(a, A, wmap, tw, s);
    case 96: return fp::WPipeLaunch<8, 12>::run(a, A, wmap, tw, s);
    case 128: return fp::WPipeLaunch<16, 8>::run(a, A, wmap, tw, s);
    case 160: return fp::WPipeLaunch<16, 10>::run(a, A, wmap, tw, s);
    case 176: return fp::WPipeLaunch<16, 11>::run(a, A, wmap, tw, s);
    case 192: return fp::WPipeLaunch<16, 12>::run(a, A, wmap, tw, s);
    case 256: return fp::WPipeLaunch<16, 16>::run(a, A, wmap, tw, s);
    default: return false;
  }
}

bool dis_fast_line(const LinePassArgs& a, const float2* tw, cudaStream_t s) {
  switch (a.N[a.axis]) {
    case 16: fp::Launch<4, 4>::line(a, tw, s); return true;
    case 32: fp::Launch<8, 4>::line(a, tw, s); return true;
    case 44: fp::Launch<4, 11>::line(a, tw, s); return true;
    case 64: fp::Launch<8, 8>::line(a, tw, s); return true;
    case 88: fp::Launch<8, 11>::line(a, tw, s); return true;
    case 96: fp::Launch<8, 12>::line(a, tw, s); return true;
    case 128: fp::Launch<16, 8>::line(a, tw, s); return true;
    case 160: fp::Launch<16, 10>::line(a, tw, s); return true;
    case 176: fp::Launch<16, 11>::line(a, tw, s); return true;
    case 192: fp::Launch<16, 12>::line(a, tw, s); return true;
    case 256: fp::Launch<16, 16>::line(a, tw, s); return true;
    default: return false;
  }
}

bool dis_fast_expand(int n, const CoilArgs& a, const float2* z, float2* A, const float2* tw, cudaStream_t s) {
  switch (n) {
    case 16: fp::Launch<4, 4>::expand(a, z, A, tw, s); return true;
    case 32: fp::Launch<8, 4>::expand(a, z, A, tw, s); return true;
    case 44: fp::Launch<4, 11>::expand(a, z, A, tw, s); return true;
    case 64: fp::Launch<8, 8>::expand(a, z, A, tw, s); return true;
    case 88: fp::Launch<8, 11>::expand(a, z, A, tw, s); return true;
    case 96: fp::Launch<8, 12>::expand(a, z, A, tw, s); return true;
    case 128: fp::Launch<16, 8>::expand(a, z, A, tw, s); return true;
    case 160: fp::Launch<16, 10>::expand(a, z, A, tw, s); return true;
    case 176: fp::Launch<16, 11>::expand(a, z, A, tw, s); return true;
    case 192: fp::Launch<16, 12>::expand(a, z, A, tw, s); return true;
    case 256: fp::Launch<16, 16>::expand(a, z, A, tw, s); return true;
    default: return false;
  }
}

bool dis_fast_combine(int n, const CoilArgs& a, const float2* A, float2* u, float scale, const float2* tw,
                      cudaStream_t s) {
  switch (n) {
    case 16: fp::Launch<4, 4>::combine(a, A, u, scale, tw, s); return true;
    case 32: fp::Launch<8, 4>::combine(a, A, u, scale, tw, s); return true;
    case 44: fp::Launch<4, 11>::combine(a, A, u, scale, tw, s); return true;
    case 64: fp::Launch<8, 8>::combine(a, A, u, scale, tw, s); return true;
    case 88: fp::Launch<8, 11>::combine(a, A, u, scale, tw, s); return true;
    case 96: fp::Launch<8, 12>::combine(a, A, u, scale, tw, s); return true;
    case 128: fp::Launch<16, 8>::combine(a, A, u, scale, tw, s); return true;
    case 160: fp::Launch<16, 10>::combine(a, A, u, scale, tw, s); return true;
    case 176: fp::Launch<16, 11>::combine(a, A, u, scale, tw, s); return true;
    case 192: fp::Launch<16, 12>::combine(a, A, u, scale, tw, s); return true;
    case 256: fp::Launch<16, 16>::combine(a, A, u, scale, tw, s); return true;
    default: return false;
  }
}

bool dis_fast_axis1(int n, int mode, const CoilArgs& a, float2* A, float2* y, const float2* ymeas, long long ld,
                    int n3off, int N3y, float scale, const float* wmap, const float* We, const float* Mb,
                    const disorder_plan_s* plan, const float2* tw, cudaStream_t s) {
  switch (n) {
    case 16: fp::Launch<4, 4>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 32: fp::Launch<8, 4>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 44: fp::Launch<4, 11>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 64: fp::Launch<8, 8>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 88: fp::Launch<8, 11>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 96: fp::Launch<8, 12>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 128: fp::Launch<16, 8>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 160: fp::Launch<16, 10>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 176: fp::Launch<16, 11>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 192: fp::Launch<16, 12>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    case 256: fp::Launch<16, 16>::axis1(mode, a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb, plan, tw, s); return true;
    default: return false;
  }
}

bool dis_fast_plane(int n1, int mode, const pl::PlaneArgs& a, const float2* tw1, const float2* tw2, int n_slots,
                    cudaStream_t s) {
  switch (n1) {
    case 16: return pl::PlaneLaunch<4, 4>::run(mode, a, tw1, tw2, n_slots, s);
    case 32: return pl::PlaneLaunch<8, 4>::run(mode, a, tw1, tw2, n_slots, s);
    case 44: return pl::PlaneLaunch<4, 11>::run(mode, a, tw1, tw2, n_slots, s);
    case 64: return pl::PlaneLaunch<8, 8>::run(mode, a, tw1, tw2, n_slots, s);
    case 88: return pl::PlaneLaunch<8, 11>::run(mode, a, tw1, tw2, n_slots, s);
    case 96: return pl::PlaneLaunch<8, 12>::run(mode, a, tw1, tw2, n_slots, s);
    case 128: return pl::PlaneLaunch<16, 8>::run(mode, a, tw1, tw2, n_slots, s);
    case 160: return pl::PlaneLaunch<16, 10>::run(mode, a, tw1, tw2, n_slots, s);
    case 176: return pl::PlaneLaunch<16, 11>::run(mode, a, tw1, tw2, n_slots, s);
    case 192: return pl::PlaneLaunch<16, 12>::run(mode, a, tw1, tw2, n_slots, s);
    case 256: return pl::PlaneLaunch<16, 16>::run(mode, a, tw1, tw2, n_slots, s);
    default: return false;
  }
}

size_t dis_plane_smem(int n1, int N2, int C, int max_ns) {
  switch (n1) {
    case 16: return pl::Layout<4, 4>::bytes(N2, C, max_ns);
    case 32: return pl::Layout<8, 4>::bytes(N2, C, max_ns);
    case 44: return pl::Layout<4, 11>::bytes(N2, C, max_ns);
    case 64: return pl::Layout<8, 8>::bytes(N2, C, max_ns);
    case 88: return pl::Layout<8, 11>::bytes(N2, C, max_ns);
    case 96: return pl::Layout<8, 12>::bytes(N2, C, max_ns);
    case 128: return pl::Layout<16, 8>::bytes(N2, C, max_ns);
    case 160: return pl::Layout<16, 10>::bytes(N2, C, max_ns);
    case 176: return pl::Layout<16, 11>::bytes(N2, C, max_ns);
    case 192: return pl::Layout<16, 12>::bytes(N2, C, max_ns);
    case 256: return pl::Layout<16, 16>::bytes(N2, C, max_ns);
    default: return (size_t)-1;
  }
}
