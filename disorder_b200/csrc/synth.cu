// Synthetic scan data on the GPU: the phantom, the coil maps and the
// measurement noise of the simulation recipe.
//
// The reference simulates its acquisitions from a ground-truth image and coil
// maps it loads from files (fig0506.m:53-56) and adds complex Gaussian noise
// (Methods/plugNoise.m:17, Simulation/synthesizeY.m:82-84). Those files are
// not distributed, so the image and coils here are new: a sum of random
// ellipsoids with a smooth random phase, and Gaussian-bump coil sensitivities
// on a sphere normalised to unit root sum of squares. The random parameters
// are drawn on the host (disorder_b200.synth_gpu, in the order of the NumPy
// recipe disorder_b200.synth) and the kernels evaluate them per voxel, so a
// 256x256x176 scan with 32 coils is built in milliseconds.
// Noise: a counter-based generator (a 64-bit mix of seed and element index
// gives two uniforms, Box-Muller gives two normals) so every element's value
// depends only on (seed, index), not on the launch shape.
#include <cmath>
#include <vector>

#include "internal.h"

namespace {

constexpr int kST = 256;

// grid coordinate i of n points on [-0.5, 0.5) (numpy linspace, endpoint=False)
DIS_D float gcoord(int i, int n) { return -0.5f + (float)i / (float)n; }

// ell: per ellipsoid 16 floats {cx, cy, cz, ax, ay, az, R00..R22, magnitude};
// ph: per phase term 5 floats {fx, fy, fz, p0, a}
__global__ void phantom_kernel(float2* __restrict__ out, int N0, int N1, int N2, const float* __restrict__ ell,
                               int n_ell, const float* __restrict__ ph, int n_ph) {
  const long long V = (long long)N0 * N1 * N2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < V; e += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(e % N0), i1 = (int)((e / N0) % N1), i2 = (int)(e / ((long long)N0 * N1));
    const float X = gcoord(i0, N0), Y = gcoord(i1, N1), Z = gcoord(i2, N2);
    float mag = 0.f;
    for (int q = 0; q < n_ell; ++q) {
      const float* p = ell + 16 * q;
      const float dx = X - p[0], dy = Y - p[1], dz = Z - p[2];
      const float u = (p[6] * dx + p[7] * dy + p[8] * dz) / p[3];
      const float v = (p[9] * dx + p[10] * dy + p[11] * dz) / p[4];
      const float w = (p[12] * dx + p[13] * dy + p[14] * dz) / p[5];
      if (u * u + v * v + w * w <= 1.0f) mag += p[15];
    }
    float phase = 0.f;
    for (int q = 0; q < n_ph; ++q) {
      const float* p = ph + 5 * q;
      phase += p[4] * cosf(6.283185307179586f * (p[0] * X + p[1] * Y + p[2] * Z) + p[3]);
    }
    float s, c;
    sincosf(phase, &s, &c);
    out[e] = make_float2(mag * c, mag * s);
  }
}

// cp: per coil 7 floats {cx, cy, cz, kx, ky, kz, phase0}; the coil values of a
// voxel are normalised by their root sum of squares
__global__ void coils_kernel(float2* __restrict__ S, int N0, int N1, int N2, int C, const float* __restrict__ cp,
                             float width) {
  const long long V = (long long)N0 * N1 * N2;
  const float inv2w2 = 1.0f / (2.0f * width * width);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < V; e += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(e % N0), i1 = (int)((e / N0) % N1), i2 = (int)(e / ((long long)N0 * N1));
    const float X = gcoord(i0, N0), Y = gcoord(i1, N1), Z = gcoord(i2, N2);
    float rss = 0.f;
    for (int c = 0; c < C; ++c) {
      const float* p = cp + 7 * c;
      const float d2 = (X - p[0]) * (X - p[0]) + (Y - p[1]) * (Y - p[1]) + (Z - p[2]) * (Z - p[2]);
      const float g = expf(-d2 * inv2w2);
      rss += g * g;
    }
    const float inv = rsqrtf(rss);
    for (int c = 0; c < C; ++c) {
      const float* p = cp + 7 * c;
      const float d2 = (X - p[0]) * (X - p[0]) + (Y - p[1]) * (Y - p[1]) + (Z - p[2]) * (Z - p[2]);
      const float g = expf(-d2 * inv2w2) * inv;
      const float ph = 6.283185307179586f * (p[3] * X + p[4] * Y + p[5] * Z) * 0.25f + p[6];
      float s, co;
      sincosf(ph, &s, &co);
      S[e + (long long)c * V] = make_float2(g * co, g * s);
    }
  }
}

// per-block sums of |out|^2 (double)
__global__ void sumsq_kernel(const float2* __restrict__ x, long long n, double* __restrict__ part) {
  __shared__ double red[kST];
  double acc = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const float2 v = x[e];
    acc += (double)v.x * v.x + (double)v.y * v.y;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = kST / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void scale_kernel(float2* __restrict__ x, long long n, float s) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    x[e] = cscale(x[e], s);
}

__global__ void noise_kernel(float2* __restrict__ y, long long n, float sigma, uint64_t seed) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    float rad, c, s;
    dis_normal2_polar(seed, e, &rad, &c, &s);
    const float2 v = y[e];
    y[e] = make_float2(v.x + sigma * rad * c, v.y + sigma * rad * s);
  }
}

}  // namespace

extern "C" {

int disorder_synth_phantom(disorder_ctx ctx, const int32_t* N, int32_t n_ell, const float* ell, int32_t n_ph,
                           const float* ph, int32_t normalise, void* out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!N || !out || n_ell < 0 || n_ph < 0 || (n_ell && !ell) || (n_ph && !ph) || N[0] < 1 || N[1] < 1 || N[2] < 1)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "synth_phantom: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  Workspace ws;
  DIS_TRY(dis_small(ctx, &ws));
  float* dp = ws.take<float>((size_t)16 * n_ell + 5 * n_ph + 1);
  if (!dp) return dis_set_error(ctx, DISORDER_OOM, "synth_phantom: too many parameters");
  if (n_ell) DIS_CUDA_TRY(cudaMemcpyAsync(dp, ell, sizeof(float) * 16 * n_ell, cudaMemcpyHostToDevice, ctx->stream));
  if (n_ph)
    DIS_CUDA_TRY(cudaMemcpyAsync(dp + 16 * n_ell, ph, sizeof(float) * 5 * n_ph, cudaMemcpyHostToDevice, ctx->stream));
  phantom_kernel<<<4 * ctx->sm_count, kST, 0, ctx->stream>>>((float2*)out, N[0], N[1], N[2], dp, n_ell,
                                                             dp + 16 * n_ell, n_ph);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  if (normalise) {  // x / ||x|| (fig0506.m:95)
    const long long V = (long long)N[0] * N[1] * N[2];
    const int nb = 2 * ctx->sm_count;
    double* part = ws.take<double>(nb);
    if (!part) return dis_set_error(ctx, DISORDER_OOM, "synth_phantom workspace");
    sumsq_kernel<<<nb, kST, 0, ctx->stream>>>((const float2*)out, V, part);
    dis_count(ctx);
    std::vector<double> h(nb);
    DIS_CUDA_TRY(cudaMemcpyAsync(h.data(), part, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream));
    DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    double tot = 0;
    for (double v : h) tot += v;
    if (tot > 0) {
      scale_kernel<<<4 * ctx->sm_count, kST, 0, ctx->stream>>>((float2*)out, V, (float)(1.0 / std::sqrt(tot)));
      dis_count(ctx);
    }
  }
  // the parameters are staged from pageable memory, so the copies are done
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

int disorder_synth_coils(disorder_ctx ctx, const int32_t* N, int32_t C, const float* cp, float width, void* out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!N || !out || !cp || C < 1 || width <= 0.f || N[0] < 1 || N[1] < 1 || N[2] < 1)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "synth_coils: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  Workspace ws;
  DIS_TRY(dis_small(ctx, &ws));
  float* dp = ws.take<float>((size_t)7 * C);
  if (!dp) return dis_set_error(ctx, DISORDER_OOM, "synth_coils: too many coils");
  DIS_CUDA_TRY(cudaMemcpyAsync(dp, cp, sizeof(float) * 7 * C, cudaMemcpyHostToDevice, ctx->stream));
  coils_kernel<<<4 * ctx->sm_count, kST, 0, ctx->stream>>>((float2*)out, N[0], N[1], N[2], C, dp, width);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

int disorder_add_noise(disorder_ctx ctx, void* y, int64_t n, float sigma, uint64_t seed) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!y || n < 0) return dis_set_error(ctx, DISORDER_BAD_ARG, "add_noise: bad arguments");
  if (n == 0) return DISORDER_OK;
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  noise_kernel<<<4 * ctx->sm_count, kST, 0, ctx->stream>>>((float2*)y, n, sigma, seed);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

}  // extern "C"
