// Common device/host helpers for libdisorder (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/disorder.h"

#define DIS_HD __host__ __device__ __forceinline__
#define DIS_D __device__ __forceinline__

DIS_HD float2 c2(float x, float y) { return make_float2(x, y); }
DIS_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
DIS_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
DIS_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
DIS_HD float2 cmulc(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }  // a*conj(b)
DIS_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
DIS_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
DIS_HD float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }   // i*a
DIS_HD float2 cmulmi(float2 a) { return make_float2(a.y, -a.x); }  // -i*a
DIS_HD float2 cfma(float2 a, float2 b, float2 acc) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y)));
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
