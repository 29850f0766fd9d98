// Line-pass kernels: every DFT-based step of the hot path is a pass over
// lines of a volume along one axis: load a tile of L lines into shared
// memory, FFT, multiply by phase factors (and combine up to two inputs),
// inverse FFT, store. One HBM read and one write of the volume per pass.
#include <algorithm>
#include <cstdlib>

#include "fastpass.h"
#include "internal.h"
#include "tiles.cuh"

namespace {

constexpr int kThreads = 256;

DIS_D float2 coef(int code, const LinePassArgs& a, int slot, const LineTile& t, int l, int k, float invn) {
  switch (code) {
    case P_A: {
      const int row = a.A.b >= 0 ? t.coord[l][a.A.b] : 0;
      return a.A.p[slot * a.A.sstride + (long long)row * a.plan.n + k];
    }
    case P_B: {
      const int row = a.B.b >= 0 ? t.coord[l][a.B.b] : 0;
      return a.B.p[slot * a.B.sstride + (long long)row * a.plan.n + k];
    }
    case P_ONE:
      return make_float2(invn, 0.f);
    case P_DK:
      return make_float2(0.f, -a.kG[k] * invn);
    default:
      return make_float2(0.f, 0.f);
  }
}

__global__ void __launch_bounds__(kThreads) line_pass_kernel(LinePassArgs a) {
  extern __shared__ float2 sm[];
  __shared__ LineTile tl;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.plan.n, L = a.L, P = a.pitch;
  const int axis = a.axis;
  float2* tw = sm;
  float2* b0 = sm + ((n + 1) & ~1);
  const long long bsz = (long long)n * P;
  float2* b1 = b0 + bsz;
  const bool two = (a.in1 != nullptr) || (a.out1 != nullptr);
  float2* b2 = b1 + bsz;
  float2* b3 = b2 + bsz;
  float2* acc = two ? b3 + bsz : b2;
  load_twiddles(tw, n, tid, nthr);
  tile_lines(a.N, axis, L, blockIdx.x, &tl, tid);
  const float invn = 1.0f / (float)n;
  int s_begin = blockIdx.y, s_end = blockIdx.y + 1;
  if (a.accumulate) {
    s_begin = 0;
    s_end = a.n_slots;
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e % L, k = e / L;
      acc[k * P + l] = make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  for (int slot = s_begin; slot < s_end; ++slot) {
    load_tile(a.in0 + slot * a.in0_s, b0, tl, a.N, axis, n, L, P, false, tid, nthr);
    if (a.in1) load_tile(a.in1 + slot * a.in1_s, b2, tl, a.N, axis, n, L, P, false, tid, nthr);
    __syncthreads();
    float2* X0 = fft_tile(b0, b1, tw, a.plan, L, P, tid, nthr);
    float2* X0s = (X0 == b0) ? b1 : b0;
    float2* X1 = nullptr;
    float2* X1s = nullptr;
    if (a.in1) {
      X1 = fft_tile(b2, b3, tw, a.plan, L, P, tid, nthr);
      X1s = (X1 == b2) ? b3 : b2;
    } else if (two) {
      X1 = b2;
      X1s = b3;
    }
    // combine: Y0 = T (P00 X0 + P01 X1), Y1 = T (P10 X0 + P11 X1); store conj for the inverse
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e % L, k = e / L;
      const float2 x0 = X0[k * P + l];
      const float2 x1 = a.in1 ? X1[k * P + l] : make_float2(0.f, 0.f);
      float2 tf = make_float2(1.f, 0.f);
      if (a.T.p) tf = a.T.p[slot * a.T.sstride + k];
      float2 y0 = cmul(coef(a.c00, a, slot, tl, l, k, invn), x0);
      if (a.c01) y0 = cadd(y0, cmul(coef(a.c01, a, slot, tl, l, k, invn), x1));
      y0 = cmul(y0, tf);
      float2 y1 = make_float2(0.f, 0.f);
      if (a.out1) {
        y1 = cmul(coef(a.c10, a, slot, tl, l, k, invn), x0);
        if (a.c11) y1 = cadd(y1, cmul(coef(a.c11, a, slot, tl, l, k, invn), x1));
        y1 = cmul(y1, tf);
      }
      X0[k * P + l] = cconj(y0);
      if (a.out1) X1[k * P + l] = cconj(y1);
    }
    __syncthreads();
    float2* Y0 = fft_tile(X0, X0s, tw, a.plan, L, P, tid, nthr);
    float2* Y1 = a.out1 ? fft_tile(X1, X1s, tw, a.plan, L, P, tid, nthr) : nullptr;
    if (a.accumulate) {
      for (int e = tid; e < n * L; e += nthr) {
        const int l = e % L, k = e / L;
        acc[k * P + l] = cadd(acc[k * P + l], cconj(Y0[k * P + l]));
      }
    } else {
      float2* o0 = a.out0 + slot * a.out0_s;
      for_tile(tl, a.N, axis, n, L, P, tid, nthr, [&](long long g, int s) { o0[g] = cconj(Y0[s]); });
      if (a.out1) {
        float2* o1 = a.out1 + slot * a.out1_s;
        for_tile(tl, a.N, axis, n, L, P, tid, nthr, [&](long long g, int s) { o1[g] = cconj(Y1[s]); });
      }
    }
    __syncthreads();
  }
  if (a.accumulate) {
    float2* o0 = a.out0;
    const float beta = a.beta;
    for_tile(tl, a.N, axis, n, L, P, tid, nthr, [&](long long g, int s) {
      float2 v = acc[s];
      if (beta != 0.f) v = cadd(v, cscale(o0[g], beta));
      o0[g] = v;
    });
  }
}

int pick_L(int n, int nbuf, int other_extent) {
  // keep the tile within ~100 KB so two or more CTAs fit per SM
  int L = kMaxL;
  while (L > 2 && (size_t)nbuf * n * (L + 1) * sizeof(float2) > 100 * 1024) L >>= 1;
  (void)other_extent;
  return L;
}


}  // namespace

bool dis_use_fast() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("DISORDER_GENERIC_FFT");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}

// DISORDER_NO_PIPE=1 keeps every pass on the one-tile-per-CTA kernels.
bool dis_use_pipe() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("DISORDER_NO_PIPE");
    v = (e && e[0] == '1') ? 0 : 1;
  }
  return v == 1;
}

int dis_line_pass(disorder_ctx_s* ctx, LinePassArgs a) {
  const int n = a.N[a.axis];
  if (a.plan.n != n) return dis_set_error(ctx, DISORDER_BAD_ARG, "line pass: plan size %d != axis size %d", a.plan.n, n);
  if (a.n_slots == 0) return DISORDER_OK;
  if (dis_use_fast() && a.tw && dis_use_pipe() && dis_fast_tma_line(ctx, a)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  if (dis_use_fast() && a.tw && dis_use_pipe() && dis_fast_pipe(a, a.tw, ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  if (dis_use_fast() && a.tw && dis_fast_line(a, a.tw, ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  const bool two = (a.in1 != nullptr) || (a.out1 != nullptr);
  const int nbuf = (two ? 4 : 2) + (a.accumulate ? 1 : 0);
  a.L = pick_L(n, nbuf, 0);
  a.pitch = a.L + 1;
  const size_t smem = (size_t)((n + 1) & ~1) * sizeof(float2) + (size_t)nbuf * n * a.pitch * sizeof(float2);
  // set once per process (thread-safe static initialisation)
  static const cudaError_t attr =
      cudaFuncSetAttribute(line_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  (void)attr;
  if (smem > 200 * 1024) return dis_set_error(ctx, DISORDER_BAD_ARG, "line pass: size %d too large", n);
  dim3 grid((unsigned)tiles_for(a.N, a.axis, a.L), a.accumulate ? 1 : (unsigned)a.n_slots);
  if (grid.x == 0 || grid.y == 0) return DISORDER_OK;
  line_pass_kernel<<<grid, kThreads, smem, ctx->stream>>>(a);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

// ---------------------------------------------------------------- flipping
namespace {

struct FlipArgs {
  int N[3];
  int axis;
  int L, pitch;
  float2* vols;
  long long vstride;
  const int* slots;
  float h1, h2;  // shifts before and after the reversal
  FFTPlan plan;
};

// out = shift(in, h): integer h -> circular index shift (shifting.m:29-37),
// otherwise the DFT phase ramp exp(-i k h) (shifting.m:38-47).
DIS_D float2* shift_tile(float2* src, float2* dst, float2* scr, float h, const FlipArgs& a,
                         const float2* tw, int tid, int nthr) {
  const int n = a.plan.n, L = a.L, P = a.pitch;
  if (h == floorf(h)) {
    const int hi = (int)h;
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e % L, p = e / L;
      int q = (p - hi) % n;
      if (q < 0) q += n;
      dst[p * P + l] = src[q * P + l];
    }
    __syncthreads();
    return dst;
  }
  // conj(FFT(conj(phase .* FFT(x))))/n
  float2* X = fft_tile(src, dst, tw, a.plan, L, P, tid, nthr);
  float2* Xs = (X == src) ? dst : src;
  const int half = n / 2;
  const double c = ceil((n + 1) / 2.0);
  for (int e = tid; e < n * L; e += nthr) {
    const int l = e % L, k = e / L;
    const int j = (k + half) % n;  // ifftshift
    const float kv = (float)((2.0 * 3.14159265358979323846 / n) * ((double)(j + 1) - c));
    double s, co;
    sincos(-(double)kv * (double)h, &s, &co);
    const float2 ph = make_float2((float)(co / n), (float)(s / n));
    X[k * P + l] = cconj(cmul(X[k * P + l], ph));
  }
  __syncthreads();
  float2* Y = fft_tile(X, Xs, tw, a.plan, L, P, tid, nthr);
  for (int e = tid; e < n * L; e += nthr) {
    const int l = e % L, k = e / L;
    Y[k * P + l] = cconj(Y[k * P + l]);
  }
  __syncthreads();
  (void)scr;
  return Y;
}

__global__ void __launch_bounds__(kThreads) flip_kernel(FlipArgs a) {
  extern __shared__ float2 sm[];
  __shared__ LineTile tl;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.plan.n, L = a.L, P = a.pitch;
  float2* tw = sm;
  float2* b0 = sm + ((n + 1) & ~1);
  float2* b1 = b0 + (long long)n * P;
  load_twiddles(tw, n, tid, nthr);
  tile_lines(a.N, a.axis, L, blockIdx.x, &tl, tid);
  __syncthreads();
  float2* v = a.vols + (long long)a.slots[blockIdx.y] * a.vstride;
  load_tile(v, b0, tl, a.N, a.axis, n, L, P, false, tid, nthr);
  __syncthreads();
  float2* r = shift_tile(b0, b1, nullptr, a.h1, a, tw, tid, nthr);
  float2* o = (r == b0) ? b1 : b0;
  for (int e = tid; e < n * L; e += nthr) {
    const int l = e % L, p = e / L;
    o[p * P + l] = r[(n - 1 - p) * P + l];  // flip (reverse the axis)
  }
  __syncthreads();
  r = shift_tile(o, r, nullptr, a.h2, a, tw, tid, nthr);
  for_tile(tl, a.N, a.axis, n, L, P, tid, nthr, [&](long long g, int s) { v[g] = r[s]; });
}

}  // namespace

int dis_flip_pass(disorder_ctx_s* ctx, const disorder_plan_s* plan, float2* vols, long long vstride,
                  const int* d_slots, int n_slots, int axis, float cent) {
  if (n_slots == 0) return DISORDER_OK;
  FlipArgs a;
  for (int i = 0; i < 3; ++i) a.N[i] = plan->N[i];
  a.axis = axis;
  const int n = plan->N[axis];
  a.L = pick_L(n, 2, 0);
  a.pitch = a.L + 1;
  a.vols = vols;
  a.vstride = vstride;
  a.slots = d_slots;
  a.h1 = -cent + 0.5f;  // flipping.m:13-15
  a.h2 = cent - 0.5f;
  a.plan = plan->fft[axis];
  const size_t smem = (size_t)((n + 1) & ~1) * sizeof(float2) + 2 * (size_t)n * a.pitch * sizeof(float2);
  static const cudaError_t attr =
      cudaFuncSetAttribute(flip_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  (void)attr;
  dim3 grid((unsigned)tiles_for(plan->N, axis, a.L), (unsigned)n_slots);
  flip_kernel<<<grid, kThreads, smem, ctx->stream>>>(a);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}
