// Learned motion proposal: a small 3-D convolutional network that maps one
// motion state's back-projected k-space residual to a 6-parameter motion
// update, with its forward, backward and Adam kernels, plus the per-state
// residual entry points it is fed by and the per-sample residual energies of
// the driver's outlier weighting. There is no counterpart in the
// reference; the plain Levenberg-Marquardt step (LMsolver.m) still decides
// on every proposal (the caller accepts a proposal only where the state's
// energy drops).
//
// Activations are channels-last, level l holding [batch][n3][n2][n1][channel]
// in FP32, so a complex volume (n1 fastest, real and imaginary interleaved)
// is level 0 with two channels exactly as it lies in memory. Weights are BF16
// (an FP32 master copy is kept for training); every sum is FP32. The network
// is about 85 M multiply-adds per 64x64x44 volume, so the kernels are plain
// CUDA-core loops: one thread per output element, lanes over output channels
// (weights coalesced, inputs broadcast), float4 channel loads.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "encoding.h"
#include "internal.h"
#include "solvers.h"

namespace {

constexpr int kConv = 4;
constexpr int kCh[kConv + 1] = {4, 16, 32, 64, 64};
constexpr int kHid = 128;
constexpr int kOut = 6;
constexpr int kMinD = 16;            // smallest input extent (keeps every level >= 1 voxel)
constexpr float kTransUnit = 2.f;    // outputs 0-2: translation / 2 (voxels of the input volume's grid)
constexpr float kRotUnitDeg = 8.f;   // outputs 3-5: rotation / 8 degrees

struct Layout {
  long long w[kConv], b[kConv], f1w, f1b, f2w, f2b, total;
};

Layout make_layout() {
  Layout L{};
  long long o = 0;
  for (int l = 0; l < kConv; ++l) {
    L.w[l] = o;
    o += 27LL * kCh[l] * kCh[l + 1];
    L.b[l] = o;
    o += kCh[l + 1];
  }
  L.f1w = o;
  o += (long long)kCh[kConv] * kHid;
  L.f1b = o;
  o += kHid;
  L.f2w = o;
  o += (long long)kHid * kOut;
  L.f2b = o;
  o += kOut;
  L.total = o;
  return L;
}

using bf16 = __nv_bfloat16;

__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }

// exact GELU, z * Phi(z), and its derivative Phi(z) + z * phi(z)
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

template <int CI>
__device__ __forceinline__ void load_ch(const float* __restrict__ p, float (&v)[CI]) {
  if constexpr (CI % 4 == 0) {
#pragma unroll
    for (int c = 0; c < CI / 4; ++c) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(p) + c);
      v[4 * c] = q.x;
      v[4 * c + 1] = q.y;
      v[4 * c + 2] = q.z;
      v[4 * c + 3] = q.w;
    }
  } else {
#pragma unroll
    for (int c = 0; c < CI; ++c) v[c] = __ldg(p + c);
  }
}

// pre = bias + in_scale * conv(in, w), act = gelu(pre); 3x3x3, stride 2,
// zero padding 1: output o reads inputs 2o-1 .. 2o+1 along each axis.
template <int CI, int CO>
__global__ void __launch_bounds__(256) conv_fwd_kernel(const float* __restrict__ in, float in_scale,
                                                       const bf16* __restrict__ w, const bf16* __restrict__ bias,
                                                       int B, int I1, int I2, int I3, int O1, int O2, int O3,
                                                       float* __restrict__ pre, float* __restrict__ act) {
  const long long total = (long long)B * O1 * O2 * O3 * CO;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int co = (int)(idx % CO);
  long long r = idx / CO;
  const int o1 = (int)(r % O1);
  r /= O1;
  const int o2 = (int)(r % O2);
  r /= O2;
  const int o3 = (int)(r % O3);
  const int b = (int)(r / O3);
  float s = 0.f;
  for (int kz = 0; kz < 3; ++kz) {
    const int i3 = 2 * o3 - 1 + kz;
    if (i3 < 0 || i3 >= I3) continue;
    for (int ky = 0; ky < 3; ++ky) {
      const int i2 = 2 * o2 - 1 + ky;
      if (i2 < 0 || i2 >= I2) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int i1 = 2 * o1 - 1 + kx;
        if (i1 < 0 || i1 >= I1) continue;
        float v[CI];
        load_ch<CI>(in + ((((long long)b * I3 + i3) * I2 + i2) * I1 + i1) * CI, v);
        const bf16* wp = w + ((kz * 3 + ky) * 3 + kx) * CI * CO + co;
#pragma unroll
        for (int c = 0; c < CI; ++c) s = fmaf(v[c], bf(wp[c * CO]), s);
      }
    }
  }
  const float z = bf(bias[co]) + in_scale * s;
  pre[idx] = z;
  act[idx] = gelu(z);
}

// The first convolution reads its 4 input channels from two complex
// volumes: channels 0-1 from the batch volume b of `in` (times s_in), channels
// 2-3 from the one volume `ref` shared by the batch (times s_ref; NULL reads
// zeros).
__device__ __forceinline__ void load_in0(const float2* __restrict__ in, float s_in, const float2* __restrict__ ref,
                                         float s_ref, long long vb, long long vi, float (&v)[4]) {
  const float2 a = __ldg(in + vb + vi);
  v[0] = s_in * a.x;
  v[1] = s_in * a.y;
  if (ref) {
    const float2 r = __ldg(ref + vi);
    v[2] = s_ref * r.x;
    v[3] = s_ref * r.y;
  } else {
    v[2] = v[3] = 0.f;
  }
}

template <int CO>
__global__ void __launch_bounds__(256) conv0_fwd_kernel(const float2* __restrict__ in, float s_in,
                                                        const float2* __restrict__ ref, float s_ref,
                                                        const bf16* __restrict__ w, const bf16* __restrict__ bias,
                                                        int B, int I1, int I2, int I3, int O1, int O2, int O3,
                                                        float* __restrict__ pre, float* __restrict__ act) {
  constexpr int CI = 4;
  const long long total = (long long)B * O1 * O2 * O3 * CO;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int co = (int)(idx % CO);
  long long r = idx / CO;
  const int o1 = (int)(r % O1);
  r /= O1;
  const int o2 = (int)(r % O2);
  r /= O2;
  const int o3 = (int)(r % O3);
  const int b = (int)(r / O3);
  const long long vb = (long long)b * I1 * I2 * I3;
  float s = 0.f;
  for (int kz = 0; kz < 3; ++kz) {
    const int i3 = 2 * o3 - 1 + kz;
    if (i3 < 0 || i3 >= I3) continue;
    for (int ky = 0; ky < 3; ++ky) {
      const int i2 = 2 * o2 - 1 + ky;
      if (i2 < 0 || i2 >= I2) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int i1 = 2 * o1 - 1 + kx;
        if (i1 < 0 || i1 >= I1) continue;
        float v[CI];
        load_in0(in, s_in, ref, s_ref, vb, ((long long)i3 * I2 + i2) * I1 + i1, v);
        const bf16* wp = w + ((kz * 3 + ky) * 3 + kx) * CI * CO + co;
#pragma unroll
        for (int c = 0; c < CI; ++c) s = fmaf(v[c], bf(wp[c * CO]), s);
      }
    }
  }
  const float z = bf(bias[co]) + s;
  pre[idx] = z;
  act[idx] = gelu(z);
}

// weight gradient of the first convolution (inputs as conv0_fwd_kernel)
template <int CO>
__global__ void __launch_bounds__(256) conv0_wgrad_kernel(const float2* __restrict__ in, float s_in,
                                                          const float2* __restrict__ ref, float s_ref,
                                                          const float* __restrict__ dout, int B, int I1, int I2,
                                                          int I3, int O1, int O2, int O3, long long rows_per,
                                                          float* __restrict__ gw) {
  constexpr int CI = 4;
  constexpr int NW = 27 * CI * CO;
  const int wi = blockIdx.x * blockDim.x + threadIdx.x;
  if (wi >= NW) return;
  const int co = wi % CO;
  const int ci = (wi / CO) % CI;
  const int tap = wi / (CO * CI);
  const int kx = tap % 3, ky = (tap / 3) % 3, kz = tap / 9;
  const bool from_ref = ci >= 2;
  if (from_ref && !ref) return;
  const float* src = reinterpret_cast<const float*>(from_ref ? ref : in) + (ci & 1);
  const float sc = from_ref ? s_ref : s_in;
  const long long rows = (long long)B * O3 * O2;
  const long long r0 = (long long)blockIdx.y * rows_per;
  const long long r1 = min(rows, r0 + rows_per);
  const int o1lo = kx == 0 ? 1 : 0;
  const int o1hi = min(O1, (I1 - kx) / 2 + 1);
  float s = 0.f;
  for (long long rr = r0; rr < r1; ++rr) {
    const int o2 = (int)(rr % O2);
    const long long q = rr / O2;
    const int o3 = (int)(q % O3);
    const int b = (int)(q / O3);
    const int i3 = 2 * o3 - 1 + kz, i2 = 2 * o2 - 1 + ky;
    if (i3 < 0 || i3 >= I3 || i2 < 0 || i2 >= I2) continue;
    const long long vrow = ((from_ref ? 0LL : (long long)b * I3) + i3) * I2 + i2;
    const float* ip = src + vrow * (long long)I1 * 2;
    const float* dp = dout + (((long long)b * O3 + o3) * O2 + o2) * (long long)O1 * CO + co;
    for (int o1 = o1lo; o1 < o1hi; ++o1) s = fmaf(__ldg(ip + (2 * o1 - 1 + kx) * 2), __ldg(dp + o1 * CO), s);
  }
  atomicAdd(gw + wi, s * sc);
}

// din = (conv^T dout) * gelu'(pre_in): the gradient with respect to the
// pre-activation of the input level. wT: [tap][CO][CI].
template <int CI, int CO>
__global__ void __launch_bounds__(256) conv_dgrad_kernel(const float* __restrict__ dout, const bf16* __restrict__ wT,
                                                         const float* __restrict__ pre_in, int B, int I1, int I2,
                                                         int I3, int O1, int O2, int O3, float* __restrict__ din) {
  const long long total = (long long)B * I1 * I2 * I3 * CI;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int ci = (int)(idx % CI);
  long long r = idx / CI;
  const int i1 = (int)(r % I1);
  r /= I1;
  const int i2 = (int)(r % I2);
  r /= I2;
  const int i3 = (int)(r % I3);
  const int b = (int)(r / I3);
  float s = 0.f;
  for (int kz = 0; kz < 3; ++kz) {
    const int t3 = i3 + 1 - kz;  // = 2 o3
    if (t3 < 0 || (t3 & 1) || (t3 >> 1) >= O3) continue;
    for (int ky = 0; ky < 3; ++ky) {
      const int t2 = i2 + 1 - ky;
      if (t2 < 0 || (t2 & 1) || (t2 >> 1) >= O2) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int t1 = i1 + 1 - kx;
        if (t1 < 0 || (t1 & 1) || (t1 >> 1) >= O1) continue;
        float d[CO];
        load_ch<CO>(dout + ((((long long)b * O3 + (t3 >> 1)) * O2 + (t2 >> 1)) * O1 + (t1 >> 1)) * CO, d);
        const bf16* wp = wT + ((kz * 3 + ky) * 3 + kx) * CO * CI + ci;
#pragma unroll
        for (int c = 0; c < CO; ++c) s = fmaf(d[c], bf(wp[c * CI]), s);
      }
    }
  }
  din[idx] = s * gelu_grad(pre_in[idx]);
}

// gw[tap][ci][co] += in_scale * sum over (b, o) of in[b][2o-1+k][ci] * dout[b][o][co];
// blockIdx.y takes rows_per rows (b, o3, o2) of the output.
template <int CI, int CO>
__global__ void __launch_bounds__(256) conv_wgrad_kernel(const float* __restrict__ in, float in_scale,
                                                         const float* __restrict__ dout, int B, int I1, int I2,
                                                         int I3, int O1, int O2, int O3, long long rows_per,
                                                         float* __restrict__ gw) {
  constexpr int NW = 27 * CI * CO;
  const int wi = blockIdx.x * blockDim.x + threadIdx.x;
  if (wi >= NW) return;
  const int co = wi % CO;
  const int ci = (wi / CO) % CI;
  const int tap = wi / (CO * CI);
  const int kx = tap % 3, ky = (tap / 3) % 3, kz = tap / 9;
  const long long rows = (long long)B * O3 * O2;
  const long long r0 = (long long)blockIdx.y * rows_per;
  const long long r1 = min(rows, r0 + rows_per);
  // o1 with 0 <= 2*o1 - 1 + kx < I1 (I1 >= 2)
  const int o1lo = kx == 0 ? 1 : 0;
  const int o1hi = min(O1, (I1 - kx) / 2 + 1);
  float s = 0.f;
  for (long long rr = r0; rr < r1; ++rr) {
    const int o2 = (int)(rr % O2);
    const long long q = rr / O2;
    const int o3 = (int)(q % O3);
    const int b = (int)(q / O3);
    const int i3 = 2 * o3 - 1 + kz, i2 = 2 * o2 - 1 + ky;
    if (i3 < 0 || i3 >= I3 || i2 < 0 || i2 >= I2) continue;
    const float* ip = in + (((long long)b * I3 + i3) * I2 + i2) * (long long)I1 * CI + ci;
    const float* dp = dout + (((long long)b * O3 + o3) * O2 + o2) * (long long)O1 * CO + co;
    for (int o1 = o1lo; o1 < o1hi; ++o1) s = fmaf(__ldg(ip + (2 * o1 - 1 + kx) * CI), __ldg(dp + o1 * CO), s);
  }
  atomicAdd(gw + wi, s * in_scale);
}

// gb[co] += sum over m of dout[m][co]; blockIdx.x takes rows m0 .. m0+per
template <int CO>
__global__ void __launch_bounds__(256) bias_grad_kernel(const float* __restrict__ dout, long long M, long long per,
                                                        float* __restrict__ gb) {
  const int co = threadIdx.x % CO;
  const int grp = threadIdx.x / CO;
  constexpr int NG = 256 / CO;
  const long long m0 = (long long)blockIdx.x * per;
  const long long m1 = min(M, m0 + per);
  float s = 0.f;
  for (long long m = m0 + grp; m < m1; m += NG) s += dout[m * CO + co];
  atomicAdd(gb + co, s);
}

// global average pool, fc1 + GELU, fc2; one block of kHid threads per sample
__global__ void __launch_bounds__(kHid) head_fwd_kernel(const float* __restrict__ act4, int nvox,
                                                        const bf16* __restrict__ w1, const bf16* __restrict__ b1,
                                                        const bf16* __restrict__ w2, const bf16* __restrict__ b2,
                                                        float* __restrict__ g, float* __restrict__ hpre,
                                                        float* __restrict__ h, float* __restrict__ out) {
  constexpr int CG = kCh[kConv];
  __shared__ float sg[CG], sh[kHid];
  const int b = blockIdx.x, t = threadIdx.x;
  if (t < CG) {
    float s = 0.f;
    for (int v = 0; v < nvox; ++v) s += act4[((long long)b * nvox + v) * CG + t];
    sg[t] = s / (float)nvox;
    g[b * CG + t] = sg[t];
  }
  __syncthreads();
  float a = bf(b1[t]);
  for (int c = 0; c < CG; ++c) a = fmaf(sg[c], bf(w1[c * kHid + t]), a);
  hpre[b * kHid + t] = a;
  const float hv = gelu(a);
  h[b * kHid + t] = hv;
  sh[t] = hv;
  __syncthreads();
  if (t < kOut) {
    float o = bf(b2[t]);
    for (int j = 0; j < kHid; ++j) o = fmaf(sh[j], bf(w2[j * kOut + t]), o);
    out[b * kOut + t] = o;
  }
}

// loss = sum (out - target)^2 / B; gradients of fc2, fc1 and the pool, then
// the gradient with respect to the last convolution's pre-activation
__global__ void __launch_bounds__(kHid) head_bwd_kernel(const float* __restrict__ target, int B,
                                                        const float* __restrict__ out, const float* __restrict__ g,
                                                        const float* __restrict__ hpre, const float* __restrict__ h,
                                                        const bf16* __restrict__ w1, const bf16* __restrict__ w2,
                                                        const float* __restrict__ pre4, int nvox,
                                                        float* __restrict__ gw1, float* __restrict__ gb1,
                                                        float* __restrict__ gw2, float* __restrict__ gb2,
                                                        float* __restrict__ dpre4, double* __restrict__ loss) {
  constexpr int CG = kCh[kConv];
  __shared__ float so[kOut], sdh[kHid], sdg[CG];
  const int b = blockIdx.x, t = threadIdx.x;
  if (t < kOut) {
    const float d = out[b * kOut + t] - target[b * kOut + t];
    so[t] = 2.f * d / (float)B;
    atomicAdd(loss, (double)d * d / B);
  }
  __syncthreads();
  const float hv = h[b * kHid + t];
  float dh = 0.f;
  for (int k = 0; k < kOut; ++k) {
    atomicAdd(gw2 + t * kOut + k, hv * so[k]);
    dh = fmaf(bf(w2[t * kOut + k]), so[k], dh);
  }
  if (t < kOut) atomicAdd(gb2 + t, so[t]);
  const float dhp = dh * gelu_grad(hpre[b * kHid + t]);
  sdh[t] = dhp;
  atomicAdd(gb1 + t, dhp);
  for (int c = 0; c < CG; ++c) atomicAdd(gw1 + c * kHid + t, g[b * CG + c] * dhp);
  __syncthreads();
  if (t < CG) {
    float dg = 0.f;
    for (int j = 0; j < kHid; ++j) dg = fmaf(bf(w1[t * kHid + j]), sdh[j], dg);
    sdg[t] = dg / (float)nvox;
  }
  __syncthreads();
  const long long base = (long long)b * nvox * CG;
  for (int e = t; e < nvox * CG; e += kHid) dpre4[base + e] = sdg[e % CG] * gelu_grad(pre4[base + e]);
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, bf16* __restrict__ wb, long long P, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  p[i] = pi;
  wb[i] = __float2bfloat16_rn(pi);
}

__global__ void to_bf16_kernel(const float* __restrict__ p, bf16* __restrict__ wb, long long P) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P) wb[i] = __float2bfloat16_rn(p[i]);
}

// wT[tap][co][ci] = w[tap][ci][co]
__global__ void transpose_kernel(const bf16* __restrict__ w, bf16* __restrict__ wT, int CI, int CO) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 27 * CI * CO) return;
  const int co = i % CO, ci = (i / CO) % CI, tap = i / (CO * CI);
  wT[(tap * CO + co) * CI + ci] = w[i];
}

// network outputs -> T units: translations times the grid spacing of each
// axis (full-grid voxels per volume voxel), rotations to radians
// out[i] = sum over readout rows and coils of wrow[n3] |r[i, n3, c]|^2
__global__ void sample_energy_kernel(const float2* __restrict__ r, long long ns, int N3, int C,
                                     const float* __restrict__ wrow, double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  double s = 0.0;
  for (int c = 0; c < C; ++c)
    for (int n3 = 0; n3 < N3; ++n3) {
      const float w = wrow ? wrow[n3] : 1.f;
      if (w == 0.f) continue;
      const float2 v = r[i + ns * (n3 + (long long)N3 * c)];
      s += (double)w * ((double)v.x * v.x + (double)v.y * v.y);
    }
  out[i] = s;
}

__global__ void convert_out_kernel(const float* __restrict__ out, int n, float sp0, float sp1, float sp2,
                                   float* __restrict__ dT) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kOut) return;
  const int s = i / kOut, k = i % kOut;
  const float u = k == 0 ? kTransUnit * sp0
                : k == 1 ? kTransUnit * sp1
                : k == 2 ? kTransUnit * sp2
                         : kRotUnitDeg * 0.017453292519943296f;
  dT[k * n + s] = out[i] * u;
}

unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace

struct disorder_net_s {
  disorder_ctx_s* ctx = nullptr;
  int L[kConv + 1][3] = {};  // spatial size of each level, level 0 = input
  int max_batch = 0;
  Layout lay{};
  float* master = nullptr;
  bf16* wb = nullptr;
  bf16* wT = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* pre[kConv + 1] = {};
  float* act[kConv + 1] = {};
  float* dbuf[2] = {};
  float* g = nullptr;
  float* hpre = nullptr;
  float* h = nullptr;
  float* out = nullptr;
  double* loss = nullptr;
  // inputs of the last forward (first convolution)
  const float2* in = nullptr;
  const float2* ref = nullptr;
  float s_in = 1.f, s_ref = 1.f;
  int batch = 0;
  std::vector<void*> allocs;
  long long vox(int l) const { return (long long)L[l][0] * L[l][1] * L[l][2]; }
};

namespace {

template <class T>
int net_alloc(disorder_net_s* n, T** p, size_t count) {
  void* q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 1)) != cudaSuccess) {
    cudaGetLastError();
    return dis_set_error(n->ctx, DISORDER_OOM, "net: device allocation of %zu bytes failed", count * sizeof(T));
  }
  n->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return DISORDER_OK;
}

int refresh_copies(disorder_net_s* n) {
  disorder_ctx_s* ctx = n->ctx;
  cudaStream_t s = n->ctx->stream;
  for (int l = 1; l < kConv; ++l)
    transpose_kernel<<<blocks(27LL * kCh[l] * kCh[l + 1]), 256, 0, s>>>(n->wb + n->lay.w[l], n->wT + n->lay.w[l],
                                                                       kCh[l], kCh[l + 1]);
  dis_count(n->ctx, kConv - 1);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int conv_fwd(disorder_net_s* n, int l, int B) {
  disorder_ctx_s* ctx = n->ctx;
  const int* I = n->L[l];
  const int* O = n->L[l + 1];
  const bf16* w = n->wb + n->lay.w[l];
  const bf16* b = n->wb + n->lay.b[l];
  const long long total = (long long)B * n->vox(l + 1) * kCh[l + 1];
  cudaStream_t s = n->ctx->stream;
  const float* in = n->act[l];
#define DIS_CONV_FWD(CI, CO)                                                                                     \
  conv_fwd_kernel<CI, CO><<<blocks(total), 256, 0, s>>>(in, 1.f, w, b, B, I[0], I[1], I[2], O[0], O[1], O[2], \
                                                         n->pre[l + 1], n->act[l + 1])
  switch (l) {
    case 0:
      conv0_fwd_kernel<16><<<blocks(total), 256, 0, s>>>(n->in, n->s_in, n->ref, n->s_ref, w, b, B, I[0], I[1], I[2],
                                                         O[0], O[1], O[2], n->pre[1], n->act[1]);
      break;
    case 1: DIS_CONV_FWD(16, 32); break;
    case 2: DIS_CONV_FWD(32, 64); break;
    default: DIS_CONV_FWD(64, 64); break;
  }
#undef DIS_CONV_FWD
  dis_count(n->ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

// gradients of convolution l from dcur (gradient at the pre-activation of
// level l+1); for l > 0 also the gradient at level l's pre-activation (dnext)
int conv_bwd(disorder_net_s* n, int l, int B, const float* dcur, float* grad, float* dnext) {
  disorder_ctx_s* ctx = n->ctx;
  const int* I = n->L[l];
  const int* O = n->L[l + 1];
  const int CI = kCh[l], CO = kCh[l + 1];
  cudaStream_t s = n->ctx->stream;
  const long long nw = 27LL * CI * CO;
  const long long rows = (long long)B * O[2] * O[1];
  const long long target = 4LL * 148 * 1024;
  const long long nchunk = std::max<long long>(1, std::min<long long>({rows, (target + nw - 1) / nw, 65535}));
  const long long rows_per = (rows + nchunk - 1) / nchunk;
  const dim3 gw(blocks(nw), (unsigned)((rows + rows_per - 1) / rows_per));
  const long long M = (long long)B * n->vox(l + 1);
  const long long bper = 4096;
  const unsigned gb = blocks(M, (int)bper);
  float* gwp = grad + n->lay.w[l];
  float* gbp = grad + n->lay.b[l];
  const long long dtotal = (long long)B * n->vox(l) * CI;
  const bf16* wT = n->wT + n->lay.w[l];
  const float* in = n->act[l];
#define DIS_CONV_BWD(CIv, COv)                                                                                     \
  conv_wgrad_kernel<CIv, COv><<<gw, 256, 0, s>>>(in, 1.f, dcur, B, I[0], I[1], I[2], O[0], O[1], O[2], rows_per, gwp); \
  bias_grad_kernel<COv><<<gb, 256, 0, s>>>(dcur, M, bper, gbp);                                                      \
  if (dnext)                                                                                                         \
    conv_dgrad_kernel<CIv, COv><<<blocks(dtotal), 256, 0, s>>>(dcur, wT, n->pre[l], B, I[0], I[1], I[2], O[0], O[1], \
                                                               O[2], dnext)
  switch (l) {
    case 0:
      conv0_wgrad_kernel<16><<<gw, 256, 0, s>>>(n->in, n->s_in, n->ref, n->s_ref, dcur, B, I[0], I[1], I[2], O[0], O[1],
                                                O[2], rows_per, gwp);
      bias_grad_kernel<16><<<gb, 256, 0, s>>>(dcur, M, bper, gbp);
      break;
    case 1: DIS_CONV_BWD(16, 32); break;
    case 2: DIS_CONV_BWD(32, 64); break;
    default: DIS_CONV_BWD(64, 64); break;
  }
#undef DIS_CONV_BWD
  dis_count(n->ctx, dnext ? 3 : 2);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int net_forward(disorder_net_s* n, const float2* in, const float2* ref, int B, float s_in, float s_ref) {
  disorder_ctx_s* ctx = n->ctx;
  n->in = in;
  n->ref = ref;
  n->s_in = s_in;
  n->s_ref = s_ref;
  for (int l = 0; l < kConv; ++l) DIS_TRY(conv_fwd(n, l, B));
  const bf16* wb = n->wb;
  head_fwd_kernel<<<B, kHid, 0, n->ctx->stream>>>(n->act[kConv], (int)n->vox(kConv), wb + n->lay.f1w,
                                                  wb + n->lay.f1b, wb + n->lay.f2w, wb + n->lay.f2b, n->g, n->hpre,
                                                  n->h, n->out);
  dis_count(n->ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  n->batch = B;
  return DISORDER_OK;
}

}  // namespace

extern "C" {

int64_t disorder_net_param_count(void) { return make_layout().total; }

int disorder_net_create(disorder_ctx ctx, const int32_t* D, int32_t max_batch, disorder_net* net) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!D || !net || max_batch < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "net: bad arguments");
  *net = nullptr;
  for (int m = 0; m < 3; ++m)
    if (D[m] < kMinD || D[m] > 1024)
      return dis_set_error(ctx, DISORDER_BAD_ARG, "net: input extent %d out of range [%d, 1024]", D[m], kMinD);
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  disorder_net_s* n = new disorder_net_s();
  n->ctx = ctx;
  n->max_batch = max_batch;
  n->lay = make_layout();
  for (int m = 0; m < 3; ++m) {
    n->L[0][m] = D[m];
    for (int l = 1; l <= kConv; ++l) n->L[l][m] = (n->L[l - 1][m] + 1) / 2;  // ceil(I/2) for k=3, s=2, p=1
  }
  const long long P = n->lay.total;
  const long long B = max_batch;
  long long dmax = 0;
  int st = DISORDER_OK;
  auto A = [&](int r) {
    if (st == DISORDER_OK) st = r;
  };
  A(net_alloc(n, &n->master, P));
  A(net_alloc(n, &n->wb, P));
  A(net_alloc(n, &n->wT, P));
  A(net_alloc(n, &n->m, P));
  A(net_alloc(n, &n->v, P));
  for (int l = 1; l <= kConv && st == DISORDER_OK; ++l) {
    const long long e = B * n->vox(l) * kCh[l];
    dmax = std::max(dmax, e);
    A(net_alloc(n, &n->pre[l], e));
    A(net_alloc(n, &n->act[l], e));
  }
  A(net_alloc(n, &n->dbuf[0], dmax));
  A(net_alloc(n, &n->dbuf[1], dmax));
  A(net_alloc(n, &n->g, B * kCh[kConv]));
  A(net_alloc(n, &n->hpre, B * kHid));
  A(net_alloc(n, &n->h, B * kHid));
  A(net_alloc(n, &n->out, B * kOut));
  A(net_alloc(n, &n->loss, 1));
  if (st == DISORDER_OK) {
    cudaMemsetAsync(n->master, 0, P * sizeof(float), ctx->stream);
    cudaMemsetAsync(n->wb, 0, P * sizeof(bf16), ctx->stream);
    cudaMemsetAsync(n->wT, 0, P * sizeof(bf16), ctx->stream);
    cudaMemsetAsync(n->m, 0, P * sizeof(float), ctx->stream);
    cudaMemsetAsync(n->v, 0, P * sizeof(float), ctx->stream);
    if (cudaGetLastError() != cudaSuccess) st = dis_set_error(ctx, DISORDER_CUDA_ERR, "net: memset failed");
  }
  if (st != DISORDER_OK) {
    disorder_net_destroy(n);
    return st;
  }
  *net = n;
  return DISORDER_OK;
}

int disorder_net_destroy(disorder_net n) {
  if (!n) return DISORDER_BAD_ARG;
  cudaSetDevice(n->ctx->device);
  cudaStreamSynchronize(n->ctx->stream);
  for (void* p : n->allocs) cudaFree(p);
  delete n;
  return DISORDER_OK;
}

#define NET_CHECK(ctx, net)                                                              \
  if (!(ctx)) return DISORDER_BAD_ARG;                                                   \
  if (!(net) || (net)->ctx != (ctx)) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad net"); \
  DIS_CUDA_TRY(cudaSetDevice((ctx)->device))

int disorder_net_set_params(disorder_ctx ctx, disorder_net net, const float* params) {
  NET_CHECK(ctx, net);
  if (!params) return dis_set_error(ctx, DISORDER_BAD_ARG, "net: null parameters");
  const long long P = net->lay.total;
  DIS_CUDA_TRY(cudaMemcpyAsync(net->master, params, P * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  to_bf16_kernel<<<blocks(P), 256, 0, ctx->stream>>>(net->master, net->wb, P);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  DIS_TRY(refresh_copies(net));
  DIS_CUDA_TRY(cudaMemsetAsync(net->m, 0, P * sizeof(float), ctx->stream));
  DIS_CUDA_TRY(cudaMemsetAsync(net->v, 0, P * sizeof(float), ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

int disorder_net_get_params(disorder_ctx ctx, disorder_net net, float* params) {
  NET_CHECK(ctx, net);
  if (!params) return dis_set_error(ctx, DISORDER_BAD_ARG, "net: null parameters");
  DIS_CUDA_TRY(cudaMemcpyAsync(params, net->master, net->lay.total * sizeof(float), cudaMemcpyDeviceToHost,
                               ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

int disorder_net_forward(disorder_ctx ctx, disorder_net net, const void* in, const void* ref, int32_t batch,
                         float in_scale, float ref_scale, float* out) {
  NET_CHECK(ctx, net);
  if (!in || batch < 1 || batch > net->max_batch)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "net forward: batch %d outside [1, %d] or null input", batch,
                         net->max_batch);
  if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(ref)) & 7)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "net forward: inputs not 8-byte aligned");
  DIS_TRY(net_forward(net, static_cast<const float2*>(in), static_cast<const float2*>(ref), batch, in_scale, ref_scale));
  if (out)
    DIS_CUDA_TRY(cudaMemcpyAsync(out, net->out, sizeof(float) * batch * kOut, cudaMemcpyDeviceToDevice, ctx->stream));
  return DISORDER_OK;
}

int disorder_net_backward(disorder_ctx ctx, disorder_net net, const float* target, int32_t batch, float* grad,
                          double* loss) {
  NET_CHECK(ctx, net);
  if (!target || !grad || batch != net->batch || !net->in)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "net backward: needs the forward of the same batch first");
  const Layout& L = net->lay;
  cudaStream_t s = ctx->stream;
  DIS_CUDA_TRY(cudaMemsetAsync(grad, 0, L.total * sizeof(float), s));
  DIS_CUDA_TRY(cudaMemsetAsync(net->loss, 0, sizeof(double), s));
  const bf16* wb = net->wb;
  float* dcur = net->dbuf[0];
  float* dnext = net->dbuf[1];
  head_bwd_kernel<<<batch, kHid, 0, s>>>(target, batch, net->out, net->g, net->hpre, net->h, wb + L.f1w, wb + L.f2w,
                                         net->pre[kConv], (int)net->vox(kConv), grad + L.f1w, grad + L.f1b,
                                         grad + L.f2w, grad + L.f2b, dcur, net->loss);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  for (int l = kConv - 1; l >= 0; --l) {
    DIS_TRY(conv_bwd(net, l, batch, dcur, grad, l > 0 ? dnext : nullptr));
    std::swap(dcur, dnext);
  }
  double lh = 0.0;
  DIS_CUDA_TRY(cudaMemcpyAsync(&lh, net->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
  DIS_CUDA_TRY(cudaStreamSynchronize(s));
  if (loss) *loss = lh;
  return DISORDER_OK;
}

int disorder_net_adam(disorder_ctx ctx, disorder_net net, const float* grad, float lr, float beta1, float beta2,
                      float eps, int32_t step) {
  NET_CHECK(ctx, net);
  if (!grad || step < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "net adam: bad arguments");
  const long long P = net->lay.total;
  const float c1 = (float)(1.0 / (1.0 - std::pow((double)beta1, step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow((double)beta2, step)));
  adam_kernel<<<blocks(P), 256, 0, ctx->stream>>>(net->master, grad, net->m, net->v, net->wb, P, lr, beta1, beta2,
                                                  eps, c1, c2);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return refresh_copies(net);
}

// ---------------------------------------------------------------- per-state residuals
static int state_range(disorder_ctx_s* ctx, const disorder_plan_s* plan, int* lo, int* hi) {
  if (*hi <= 0) {
    *lo = 0;
    *hi = plan->N[2];
  }
  if (*lo < 0 || *hi > plan->N[2] || *lo >= *hi) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad readout range");
  return DISORDER_OK;
}

static float2* residual_buffer(disorder_ctx_s* ctx, const disorder_plan_s* plan, int C, size_t extra,
                               Workspace* ws) {
  const size_t ny = (size_t)plan->n_samples * plan->N[2] * C;
  if (dis_workspace2(ctx, ny * sizeof(float2) + extra + (1 << 20), ws) != DISORDER_OK) return nullptr;
  return ws->take<float2>(ny);
}

int disorder_state_energies(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf, int32_t n_coils,
                            const void* x, const float* T, int32_t n3_lo, int32_t n3_hi, double* En) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!plan || plan->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan");
  if (!y || !Sf || !x || !En || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "state energies: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  int lo = n3_lo, hi = n3_hi;
  DIS_TRY(state_range(ctx, plan, &lo, &hi));
  const int S = plan->n_mot;
  Workspace sw;
  float2* r = residual_buffer(ctx, plan, n_coils, 0, &sw);
  if (!r) return dis_set_error(ctx, DISORDER_OOM, "state energies: no residual buffer");
  DIS_TRY(dis_state_residual(ctx, plan, (const float2*)y, (const float2*)Sf, n_coils, (const float2*)x, T, lo, hi, r));
  if (S == 0) return DISORDER_OK;
  std::vector<int> st(S);
  for (int s = 0; s < S; ++s) st[s] = s;
  Workspace w;
  DIS_TRY(dis_workspace(ctx, (size_t)S * (64 + 28) * sizeof(double) + (1 << 16), &w));
  int* d_seg = nullptr;
  DIS_TRY(dis_upload_ints(ctx, &w, st, &d_seg));
  double* d_out = w.take<double>((size_t)S * 28);
  if (!d_out) return dis_set_error(ctx, DISORDER_OOM, "state energies: workspace");
  DIS_TRY(dis_seg_sums(ctx, plan, d_seg, S, r, nullptr, 0, plan->n_samples, lo, hi - lo, plan->N[2], n_coils, nullptr,
                       d_out, &w));
  std::vector<double> sums((size_t)S * 28);
  DIS_CUDA_TRY(cudaMemcpyAsync(sums.data(), d_out, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const double NElY = (double)plan->n_samples * plan->N[2] * n_coils;
  for (int s = 0; s < S; ++s) En[s] = sums[(size_t)s * 28] / NElY;
  return DISORDER_OK;
}

// per-sample weighted residual energies of r into the host array En (d_en: device scratch)
static int sample_energies_of(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* r, int C,
                              const float* wrow, double* d_en, double* En) {
  const long long ns = plan->n_samples;
  sample_energy_kernel<<<blocks(ns), 256, 0, ctx->stream>>>(r, ns, plan->N[2], C, wrow, d_en);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  DIS_CUDA_TRY(cudaMemcpyAsync(En, d_en, sizeof(double) * ns, cudaMemcpyDeviceToHost, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

int disorder_sample_energies(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf, int32_t n_coils,
                             const void* x, const float* T, const float* Mbe, double* En) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!plan || plan->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan");
  if (!y || !Sf || !x || !En || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "sample energies: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  const long long ns = plan->n_samples;
  Workspace sw;
  float2* r = residual_buffer(ctx, plan, n_coils, ns * sizeof(double) + 256, &sw);
  double* d_en = sw.take<double>(std::max<long long>(ns, 1));
  if (!r || !d_en) return dis_set_error(ctx, DISORDER_OOM, "sample energies: no residual buffer");
  EncodeSpec sp;
  sp.x = (const float2*)x;
  sp.Sf = (const float2*)Sf;
  sp.C = n_coils;
  sp.T = T;
  sp.T_n = plan->n_mot;
  for (int s = 0; s < plan->n_seg; ++s) sp.segs.push_back(s);
  sp.n3_lo = 0;
  sp.N3c = plan->N[2];
  sp.y_ld = ns;
  sp.y_n3off = 0;
  sp.y_N3 = plan->N[2];
  DIS_TRY(dis_encode_segments(ctx, plan, sp, r, (const float2*)y));
  if (ns == 0) return DISORDER_OK;
  return sample_energies_of(ctx, plan, r, n_coils, Mbe, d_en, En);
}

int disorder_residual_energies(disorder_ctx ctx, disorder_plan plan, const void* r, int32_t n_coils, const float* Mbe,
                               double* En) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!plan || plan->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan");
  if (!r || !En || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "residual energies: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  const long long ns = plan->n_samples;
  if (ns == 0) return DISORDER_OK;
  Workspace w;
  DIS_TRY(dis_small(ctx, &w));
  double* d_en = w.take<double>(ns);
  if (!d_en) return dis_set_error(ctx, DISORDER_OOM, "residual energies: %lld samples exceed the scratch", ns);
  return sample_energies_of(ctx, plan, (const float2*)r, n_coils, Mbe, d_en, En);
}

int disorder_backproject_states(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                                int32_t n_coils, const void* x, const float* T, int32_t n3_lo, int32_t n3_hi,
                                void* out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!plan || plan->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan");
  if (!y || !Sf || !x || !out || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "back-projection: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  int lo = n3_lo, hi = n3_hi;
  DIS_TRY(state_range(ctx, plan, &lo, &hi));
  Workspace sw;
  float2* r = residual_buffer(ctx, plan, n_coils, 0, &sw);
  if (!r) return dis_set_error(ctx, DISORDER_OOM, "back-projection: no residual buffer");
  DIS_TRY(dis_state_residual(ctx, plan, (const float2*)y, (const float2*)Sf, n_coils, (const float2*)x, T, lo, hi, r));
  return dis_backproject_states(ctx, plan, r, (const float2*)Sf, n_coils, T, (float2*)out);
}

int disorder_propose_motion(disorder_ctx ctx, disorder_plan plan, disorder_net net, const void* y, const void* Sf,
                            int32_t n_coils, const void* x, const float* T, int32_t n3_lo, int32_t n3_hi, float gain,
                            float* dT) {
  NET_CHECK(ctx, net);
  if (!plan || plan->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan");
  if (!y || !Sf || !x || !dT || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "propose: bad arguments");
  for (int m = 0; m < 3; ++m)
    if (plan->N[m] != net->L[0][m])
      return dis_set_error(ctx, DISORDER_BAD_ARG, "propose: plan volume %dx%dx%d differs from the network input",
                           plan->N[0], plan->N[1], plan->N[2]);
  int lo = n3_lo, hi = n3_hi;
  DIS_TRY(state_range(ctx, plan, &lo, &hi));
  const int S = plan->n_mot;
  if (S == 0) return DISORDER_OK;
  const long long V = plan->V;
  Workspace sw;
  const size_t featb = (size_t)S * V * sizeof(float2) + (size_t)S * kOut * 2 * sizeof(float) + 1024;
  float2* r = residual_buffer(ctx, plan, n_coils, featb, &sw);
  float2* feat = sw.take<float2>((size_t)S * V);
  float* outs = sw.take<float>((size_t)S * kOut);
  float* dTd = sw.take<float>((size_t)S * kOut);
  if (!r || !feat || !outs || !dTd) return dis_set_error(ctx, DISORDER_OOM, "propose: workspace");
  double nx = 0.0;
  DIS_TRY(dis_weighted_norm(ctx, (const float2*)x, nullptr, V, &nx));
  const double rms = std::sqrt(nx / (double)V);
  if (!(rms > 0.0)) {
    std::fill(dT, dT + (size_t)6 * S, 0.f);
    return DISORDER_OK;
  }
  DIS_TRY(dis_state_residual(ctx, plan, (const float2*)y, (const float2*)Sf, n_coils, (const float2*)x, T, lo, hi, r));
  DIS_TRY(dis_backproject_states(ctx, plan, r, (const float2*)Sf, n_coils, T, feat));
  const float sc = (float)(gain / rms);
  for (int b0 = 0; b0 < S; b0 += net->max_batch) {
    const int nb = std::min(net->max_batch, S - b0);
    DIS_TRY(net_forward(net, feat + (long long)b0 * V, (const float2*)x, nb, sc, (float)(1.0 / rms)));
    DIS_CUDA_TRY(cudaMemcpyAsync(outs + (size_t)b0 * kOut, net->out, sizeof(float) * nb * kOut,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
  }
  float sp[3];
  for (int m = 0; m < 3; ++m) sp[m] = plan->rG[m][1] - plan->rG[m][0];  // rG = (N/Nres)((1:Nres) - cent)
  convert_out_kernel<<<blocks((long long)S * kOut), 256, 0, ctx->stream>>>(outs, S, sp[0], sp[1], sp[2], dTd);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  DIS_CUDA_TRY(cudaMemcpyAsync(dT, dTd, sizeof(float) * S * kOut, cudaMemcpyDeviceToHost, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  net->in = nullptr;  // the features live in the solver workspace; no backward of this forward
  return DISORDER_OK;
}

}  // extern "C"
