// Common device/host helpers for libdisorder (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/disorder.h"

#define DIS_HD __host__ __device__ __forceinline__
#define DIS_D __device__ __forceinline__

// Device-side index checks. dis_index_ok is false when i lies outside
// [0, n): it records `site` in err[1] (the context's device error word; the
// first failing site wins) and the caller skips the access, so a bad index
// never reaches memory. disorder_synchronize reports it as BAD_ARG. Indices
// that come from the caller are always checked; DIS_DEBUG_INDEX checks the
// library's own (plan-derived) indices only in a -DDISORDER_CHECKS build.
enum DisCheckSite { DIS_SITE_GATHER_ROWS = 1, DIS_SITE_WEIGHT_MAP = 2, DIS_SITE_TMA_SAMPLES = 3 };
__device__ __forceinline__ bool dis_index_ok(long long i, long long n, int* err, int site) {
  if (i >= 0 && i < n) return true;
  if (err) atomicCAS(err + 1, 0, site);
  return false;
}
#ifdef DISORDER_CHECKS
#define DIS_DEBUG_INDEX(i, n, err, site) dis_index_ok((i), (n), (err), (site))
#else
#define DIS_DEBUG_INDEX(i, n, err, site) true
#endif

DIS_HD float2 c2(float x, float y) { return make_float2(x, y); }
// Complex add/subtract. On sm_100 one packed add.f32x2 / sub.f32x2 does both
// lanes (round-to-nearest per lane, the same results as two scalar ops).
DIS_HD float2 cadd(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "add.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
DIS_HD float2 csub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// acc + a * s on both lanes: one packed fma.rn.f32x2 on sm_100, per lane the
// same single rounding as fmaf.
DIS_HD float2 cfmas(float2 a, float s, float2 acc) {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
  float2 r;
  asm("{\n\t.reg .b64 pa, ps, pc, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 ps, {%4, %4};\n\t"
      "mov.b64 pc, {%5, %6};\n\tfma.rn.f32x2 pd, pa, ps, pc;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(s), "f"(acc.x), "f"(acc.y));
  return r;
#else
  return make_float2(fmaf(a.x, s, acc.x), fmaf(a.y, s, acc.y));
#endif
}
DIS_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
DIS_HD float2 cmulc(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }  // a*conj(b)
DIS_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
DIS_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
DIS_HD float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }   // i*a
DIS_HD float2 cmulmi(float2 a) { return make_float2(a.y, -a.x); }  // -i*a
DIS_HD float2 cfma(float2 a, float2 b, float2 acc) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y)));
}

// Counter-based normal variates: the SplitMix64 finaliser of (seed, index)
// gives two 32-bit uniforms, Box-Muller turns them into two independent
// standard normals that depend only on (seed, e).
DIS_D uint64_t dis_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// (radius, cos, sin) of the pair; the normals are rad * c and rad * s
DIS_D void dis_normal2_polar(uint64_t seed, long long e, float* rad, float* c, float* s) {
  const uint64_t r = dis_mix64(seed * 0x9E3779B97F4A7C15ull + (uint64_t)e);
  const float u1 = ((float)(uint32_t)(r >> 32) + 1.0f) * 2.3283064365386963e-10f;  // (0, 1]
  const float u2 = (float)(uint32_t)r * 2.3283064365386963e-10f;                   // [0, 1)
  *rad = sqrtf(-2.0f * logf(u1));
  sincospif(2.0f * u2, s, c);
}

// Status plumbing shared by the host-side orchestration code.
#define DIS_CUDA_TRY(call)                                                   \
  do {                                                                       \
    cudaError_t e__ = (call);                                                \
    if (e__ != cudaSuccess) {                                                \
      return dis_set_error(ctx, DISORDER_CUDA_ERR, "%s:%d %s: %s", __FILE__, \
                           __LINE__, #call, cudaGetErrorString(e__));        \
    }                                                                        \
  } while (0)

#define DIS_TRY(call)                \
  do {                               \
    int s__ = (call);                \
    if (s__ != DISORDER_OK) return s__; \
  } while (0)

struct disorder_ctx_s;
int dis_set_error(disorder_ctx_s* ctx, int status, const char* fmt, ...);
