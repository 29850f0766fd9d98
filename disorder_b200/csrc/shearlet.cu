// The shearlet regularizer of the compressed-sensing reconstruction on the
// device: computeShearlet (Reconstruction/CSsolver.m:91-101), the shearlet
// branch of Reconstruction/regularize.m:27-46 and the two trace estimates of
// Reconstruction/traceEstimation.m:61-102.
//
// A 3-D shearlet of the system built by Shearlets/buildShearlet.m is the
// product of two 2-D shearlets over different dimension pairs
// (buildShearlet.m:136-146): pair 0 = dims (1,2), pair 1 = dims (1,3),
// pair 2 = dims (3,2). The device keeps only the 2-D planes (a few MB at
// 256x256x176 against 4.6 GB for the 50 complex 3-D filters) and evaluates
// S_w(k) = A(k_a, k_b) B(k_c, k_d) where a pass needs it.
//
// Every operator is a chain of DFT passes along one axis over tiles of
// lines in shared memory (fft.cuh, Stockham, any length whose factors are
// 2, 3, 5, 7, 11 or 13). The element-wise steps ride on the first pass's
// load (conj(S_w) .*, coil map .*) and the last pass's store (We .*, the
// coefficient |.|, the accumulation S_w .* into the regularizer's sum, the
// trace sums), so one filter costs 3 passes (coefficients, trace) or 6
// (regularizer) over the volume.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fastpass.h"
#include "shearlet.cuh"

namespace {

using namespace shl;

__global__ void __launch_bounds__(kThr) sh_pass_kernel(ShArgs a) {
  extern __shared__ float2 sm[];
  __shared__ LineTile tl;
  __shared__ double red[kThr / 32];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.plan.n, L = a.L, P = a.P, axis = a.axis;
  float2* tw = sm;
  float2* b0 = sm + ((n + 1) & ~1);
  float2* b1 = b0 + (long long)n * P;
  load_twiddles(tw, n, tid, nthr);
  tile_lines(a.N, axis, L, blockIdx.x, &tl, tid);
  __syncthreads();
  auto coords = [&](int s, int& c0, int& c1, int& c2) {
    const int p = s / P, l = s - p * P;
    c0 = tl.coord[l][0];
    c1 = tl.coord[l][1];
    c2 = tl.coord[l][2];
    if (axis == 0) c0 = p;
    else if (axis == 1) c1 = p;
    else c2 = p;
  };
  // lines past the volume in a partial tile are never stored; zero them so
  // the tile's FFT reads defined values
  for (int e = tid; e < n * L; e += nthr) {
    const int l = e % L;
    if (!tl.valid[l]) b0[(e / L) * P + l] = make_float2(0.f, 0.f);
  }
  for_tile(tl, a.N, axis, n, L, P, tid, nthr, [&](long long g, int s) {
    float2 v = a.in_real ? make_float2(a.in_real[g], 0.f) : a.in[g];
    if (a.pre == PRE_CONJ_FILTER) {
      int c0, c1, c2;
      coords(s, c0, c1, c2);
      v = cmul(v, cconj(filter_at(a.f, c0, c1, c2, a.N)));
    } else if (a.pre == PRE_COIL) {
      v = cmul(v, a.pre_c[g]);
    }
    b0[s] = a.inv ? cconj(v) : v;
  });
  __syncthreads();
  const float2* X = fft_tile(b0, b1, tw, a.plan, L, P, tid, nthr);
  const float invn = 1.0f / (float)n;
  bool inv = a.inv;
  if (a.mid_we) {
    // X holds conj(n IDFT(v)); the forward DFT's input is IDFT(v) .* We
    float2* Xw = const_cast<float2*>(X);
    for_tile(tl, a.N, axis, n, L, P, tid, nthr,
             [&](long long g, int s) { Xw[s] = cscale(cconj(Xw[s]), invn * a.mid_we[g]); });
    __syncthreads();
    X = fft_tile(Xw, Xw == b0 ? b1 : b0, tw, a.plan, L, P, tid, nthr);
    inv = false;
  }
  double part = 0.0;
  for_tile(tl, a.N, axis, n, L, P, tid, nthr, [&](long long g, int s) {
    float2 v = X[s];
    if (inv) v = cscale(cconj(v), invn);
    switch (a.post) {
      case POST_STORE: a.out[g] = v; break;
      case POST_TIMES_WE: a.out[g] = cscale(v, a.we[g]); break;
      case POST_COEF: {
        const float m = hypotf(v.x, v.y) + a.eps;
        a.we_out[g] = a.pw == -1.f ? 1.f / m : powf(m, a.pw);
        break;
      }
      case POST_ACC_FILTER: {
        int c0, c1, c2;
        coords(s, c0, c1, c2);
        a.acc[g] = cadd(a.acc[g], cmul(filter_at(a.f, c0, c1, c2, a.N), v));
        break;
      }
      case POST_TRACE_WE: part += (double)a.we[g] * ((double)v.x * v.x + (double)v.y * v.y); break;
      case POST_TRACE_GRID: {
        int c0, c1, c2;
        coords(s, c0, c1, c2);
        part += (double)a.scale * a.wgrid[c0 + a.N[0] * c1] * ((double)v.x * v.x + (double)v.y * v.y);
        break;
      }
      default: {
        float2 o = cscale(v, a.scale);
        if (a.beta != 0.f) o = cadd(o, cscale(a.out[g], a.beta));
        a.out[g] = o;
      }
    }
  });
  if (a.post == POST_TRACE_WE || a.post == POST_TRACE_GRID) {
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) {
      double t = 0;
      for (int w = 0; w < kThr / 32; ++w) t += red[w];
      atomicAdd(a.sum, t);
    }
  }
}

int sh_pass(disorder_ctx_s* ctx, ShArgs a) {
  const int n = a.N[a.axis];
  const int kind = fast_kind(a);
  if (dis_use_fast() && kind >= 0 && (sh_fast_a(ctx, a, kind) || sh_fast_b(ctx, a, kind))) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  if (!dis_make_fft_plan(n, &a.plan))
    return dis_set_error(ctx, DISORDER_UNSUPPORTED_FIELD, "shearlet: length %d has a prime factor above 13", n);
  a.L = 16;
  while (a.L > 2 && (size_t)2 * n * (a.L + 1) * sizeof(float2) > 100 * 1024) a.L >>= 1;
  a.P = a.L + 1;
  const size_t smem = (size_t)((n + 1) & ~1) * sizeof(float2) + (size_t)2 * n * a.P * sizeof(float2);
  // set once per process; the static's initialisation is thread-safe (host
  // threads of several contexts launch concurrently)
  static const cudaError_t attr =
      cudaFuncSetAttribute(sh_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  (void)attr;
  if (smem > 200 * 1024) return dis_set_error(ctx, DISORDER_UNSUPPORTED_FIELD, "shearlet: length %d too large", n);
  const size_t grid = tiles_for(a.N, a.axis, a.L);
  if (grid == 0) return DISORDER_OK;
  sh_pass_kernel<<<(unsigned)grid, kThr, smem, ctx->stream>>>(a);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

ShArgs base(const int* N, int axis, int inv) {
  ShArgs a;
  for (int m = 0; m < 3; ++m) a.N[m] = N[m];
  a.axis = axis;
  a.inv = inv;
  return a;
}

// a pass of a shearlet operator: the system's grid and twiddle table
ShArgs base(const disorder_shearlet_s* sh, int axis, int inv) {
  ShArgs a = base(sh->N, axis, inv);
  a.twg = sh->tw[axis];
  return a;
}

ShFilt filt(const disorder_shearlet_s* sh, int w) {
  const int* t = &sh->table[4 * w];
  ShFilt f;
  f.pa = t[0];
  f.pb = t[2];
  f.A = sh->planes + sh->pair_off[t[0]] + (long long)t[1] * sh->plane_size[t[0]];
  f.B = sh->planes + sh->pair_off[t[2]] + (long long)t[3] * sh->plane_size[t[2]];
  return f;
}

// out = DFT3(x) (x complex, or real when xr is given); with PRE_COIL the
// first pass multiplies by the coil map c.
int dft3(disorder_ctx_s* ctx, const disorder_shearlet_s* sh, const float2* x, const float* xr, float2* out) {
  for (int m = 0; m < 3; ++m) {
    ShArgs a = base(sh, m, 0);
    a.in = m == 0 ? x : out;
    a.in_real = m == 0 ? xr : nullptr;
    a.out = out;
    DIS_TRY(sh_pass(ctx, a));
  }
  return DISORDER_OK;
}

// t = IDFT3(conj(S_w) .* xF) with the last pass's store given by `last`
int filtered_inverse(disorder_ctx_s* ctx, const disorder_shearlet_s* sh, int w, const float2* xF, float2* t,
                     const ShArgs& last) {
  for (int m = 0; m < 3; ++m) {
    ShArgs a = m == 2 ? last : base(sh, m, 1);
    a.axis = m;
    a.inv = 1;
    a.in = m == 0 ? xF : t;
    a.out = t;
    if (m == 0) {
      a.pre = PRE_CONJ_FILTER;
      a.f = filt(sh, w);
    }
    DIS_TRY(sh_pass(ctx, a));
  }
  return DISORDER_OK;
}

int check_sh(disorder_ctx ctx, disorder_shearlet sh) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!sh || sh->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "shearlet: system of another context");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  return DISORDER_OK;
}

int read_sum(disorder_ctx_s* ctx, const double* d, double* h) {
  DIS_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

}  // namespace

int disorder_shearlet_create(disorder_ctx ctx, const int32_t N[3], int32_t n_planes, const void* planes0,
                             const void* planes1, const void* planes2, int32_t n_filters, const int32_t* table,
                             disorder_shearlet* out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!N || !out || !planes0 || !planes1 || !planes2 || !table || n_planes < 1 || n_filters < 1)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "shearlet_create: bad arguments");
  *out = nullptr;
  for (int m = 0; m < 3; ++m) {
    FFTPlan p;
    if (N[m] < 1 || !dis_make_fft_plan(N[m], &p))
      return dis_set_error(ctx, DISORDER_UNSUPPORTED_FIELD, "shearlet_create: size %d is not a product of 2, 3, 5, 7, "
                           "11 and 13", N[m]);
  }
  for (int w = 0; w < n_filters; ++w)
    for (int h = 0; h < 2; ++h) {
      const int q = table[4 * w + 2 * h], k = table[4 * w + 2 * h + 1];
      if (q < 0 || q > 2 || k < 0 || k >= n_planes)
        return dis_set_error(ctx, DISORDER_BAD_ARG, "shearlet_create: table row %d names pair %d plane %d", w, q, k);
    }
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  auto* sh = new disorder_shearlet_s;
  sh->ctx = ctx;
  for (int m = 0; m < 3; ++m) sh->N[m] = N[m];
  sh->n_planes = n_planes;
  sh->n_filters = n_filters;
  sh->table.assign(table, table + 4 * n_filters);
  long long tot = 0;
  for (int q = 0; q < 3; ++q) {
    sh->pair_off[q] = tot;
    sh->plane_size[q] = (long long)N[kPair[q][0]] * N[kPair[q][1]];
    tot += sh->plane_size[q] * n_planes;
  }
  if (cudaMalloc(&sh->planes, sizeof(float2) * tot) != cudaSuccess) {
    cudaGetLastError();
    delete sh;
    return dis_set_error(ctx, DISORDER_OOM, "shearlet_create: planes");
  }
  for (int m = 0; m < 3; ++m) {
    std::vector<float2> w(N[m]);
    for (int k = 0; k < N[m]; ++k) {
      const double ang = -2.0 * 3.14159265358979323846 * (double)k / (double)N[m];
      w[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    if (cudaMalloc(&sh->tw[m], sizeof(float2) * N[m]) != cudaSuccess ||
        cudaMemcpy(sh->tw[m], w.data(), sizeof(float2) * N[m], cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      for (int q = 0; q <= m; ++q) cudaFree(sh->tw[q]);
      cudaFree(sh->planes);
      delete sh;
      return dis_set_error(ctx, DISORDER_OOM, "shearlet_create: twiddle tables");
    }
  }
  const void* src[3] = {planes0, planes1, planes2};
  for (int q = 0; q < 3; ++q) {
    const cudaError_t e = cudaMemcpy(sh->planes + sh->pair_off[q], src[q], sizeof(float2) * sh->plane_size[q] * n_planes,
                                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(sh->planes);
      for (int m = 0; m < 3; ++m) cudaFree(sh->tw[m]);
      delete sh;
      return dis_set_error(ctx, DISORDER_CUDA_ERR, "shearlet_create: %s", cudaGetErrorString(e));
    }
  }
  *out = sh;
  return DISORDER_OK;
}

int disorder_shearlet_destroy(disorder_shearlet sh) {
  if (!sh) return DISORDER_BAD_ARG;
  cudaSetDevice(sh->ctx->device);
  cudaStreamSynchronize(sh->ctx->stream);
  cudaFree(sh->planes);
  for (int m = 0; m < 3; ++m) cudaFree(sh->tw[m]);
  delete sh;
  return DISORDER_OK;
}

int disorder_shearlet_coefficients(disorder_ctx ctx, disorder_shearlet sh, const void* x, float eps, float pw,
                                   float* We) {
  DIS_TRY(check_sh(ctx, sh));
  if (!x || !We) return dis_set_error(ctx, DISORDER_BAD_ARG, "shearlet_coefficients: bad arguments");
  const long long V = (long long)sh->N[0] * sh->N[1] * sh->N[2];
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, sizeof(float2) * 2 * V + 1024, &ws));
  float2* xF = ws.take<float2>(V);
  float2* t = ws.take<float2>(V);
  DIS_TRY(dft3(ctx, sh, (const float2*)x, nullptr, xF));
  for (int w = 0; w < sh->n_filters; ++w) {
    ShArgs last = base(sh, 2, 1);
    last.post = POST_COEF;
    last.we_out = We + (long long)w * V;
    last.eps = eps;
    last.pw = pw;
    DIS_TRY(filtered_inverse(ctx, sh, w, xF, t, last));
  }
  return DISORDER_OK;
}

// out = beta out + scale IDFT3(sum_w S_w .* DFT3(We_w .* IDFT3(conj(S_w) .* DFT3(x))))
int dis_shearlet_regularize(disorder_ctx_s* ctx, const disorder_shearlet_s* sh, const float2* x, const float* We,
                            float scale, float beta, float2* out) {
  const long long V = (long long)sh->N[0] * sh->N[1] * sh->N[2];
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, sizeof(float2) * 3 * V + 1024, &ws));
  float2* xF = ws.take<float2>(V);
  float2* t = ws.take<float2>(V);
  float2* acc = ws.take<float2>(V);
  DIS_TRY(dft3(ctx, sh, x, nullptr, xF));
  DIS_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(float2) * V, ctx->stream));
  for (int w = 0; w < sh->n_filters; ++w) {
    // inverse along dims 1-2 (conj(S_w) on the first load); along dim 3 the
    // inverse, We_w and the forward DFT in one pass; forward along dims 2, 1
    // with S_w .* accumulated on the last store: 5 passes per shearlet
    ShArgs mid = base(sh, 2, 1);
    mid.mid_we = We + (long long)w * V;
    DIS_TRY(filtered_inverse(ctx, sh, w, xF, t, mid));
    for (int m = 1; m >= 0; --m) {
      ShArgs a = base(sh, m, 0);
      a.in = t;
      a.out = t;
      if (m == 0) {
        a.post = POST_ACC_FILTER;
        a.acc = acc;
        a.f = filt(sh, w);
      }
      DIS_TRY(sh_pass(ctx, a));
    }
  }
  for (int m = 0; m < 3; ++m) {
    ShArgs a = base(sh, m, 1);
    a.in = acc;
    a.out = m == 2 ? out : acc;
    if (m == 2) {
      a.post = POST_AXPBY;
      a.scale = scale;
      a.beta = beta;
    }
    DIS_TRY(sh_pass(ctx, a));
  }
  return DISORDER_OK;
}

int disorder_shearlet_regularize(disorder_ctx ctx, disorder_shearlet sh, const void* x, const float* We, float scale,
                                 float beta, void* out) {
  DIS_TRY(check_sh(ctx, sh));
  if (!x || !We || !out) return dis_set_error(ctx, DISORDER_BAD_ARG, "shearlet_regularize: bad arguments");
  return dis_shearlet_regularize(ctx, sh, (const float2*)x, We, scale, beta, (float2*)out);
}

int disorder_shearlet_trace(disorder_ctx ctx, disorder_shearlet sh, const float* probe, const float* We, double* tr) {
  DIS_TRY(check_sh(ctx, sh));
  if (!probe || !We || !tr) return dis_set_error(ctx, DISORDER_BAD_ARG, "shearlet_trace: bad arguments");
  const long long V = (long long)sh->N[0] * sh->N[1] * sh->N[2];
  Workspace ws, sw;
  DIS_TRY(dis_workspace(ctx, sizeof(float2) * 2 * V + 1024, &ws));
  DIS_TRY(dis_small(ctx, &sw));
  float2* xF = ws.take<float2>(V);
  float2* t = ws.take<float2>(V);
  double* sum = sw.take<double>(1);
  DIS_CUDA_TRY(cudaMemsetAsync(sum, 0, sizeof(double), ctx->stream));
  DIS_TRY(dft3(ctx, sh, nullptr, probe, xF));
  for (int w = 0; w < sh->n_filters; ++w) {
    ShArgs last = base(sh, 2, 1);
    last.post = POST_TRACE_WE;
    last.we = We + (long long)w * V;
    last.sum = sum;
    DIS_TRY(filtered_inverse(ctx, sh, w, xF, t, last));
  }
  return read_sum(ctx, sum, tr);
}

int disorder_fidelity_trace(disorder_ctx ctx, const int32_t N[3], const float* probe, const void* Sf, int32_t C,
                            const float* wgrid, double* tr) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!N || !probe || !Sf || C < 1 || !wgrid || !tr)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "fidelity_trace: bad arguments");
  for (int m = 0; m < 2; ++m) {
    FFTPlan p;
    if (N[m] < 1 || !dis_make_fft_plan(N[m], &p))
      return dis_set_error(ctx, DISORDER_UNSUPPORTED_FIELD, "fidelity_trace: size %d is not a product of 2, 3, 5, 7, "
                           "11 and 13", N[m]);
  }
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  const int Nv[3] = {N[0], N[1], N[2]};
  const long long V = (long long)N[0] * N[1] * N[2];
  Workspace ws, sw;
  DIS_TRY(dis_workspace(ctx, sizeof(float2) * V + 1024, &ws));
  DIS_TRY(dis_small(ctx, &sw));
  float2* t = ws.take<float2>(V);
  double* sum = sw.take<double>(1);
  DIS_CUDA_TRY(cudaMemsetAsync(sum, 0, sizeof(double), ctx->stream));
  for (int c = 0; c < C; ++c) {
    ShArgs a = base(Nv, 0, 0);  // DFT along dim 1 of S_c .* probe
    a.in_real = probe;
    a.pre = PRE_COIL;
    a.pre_c = (const float2*)Sf + (long long)c * V;
    a.out = t;
    DIS_TRY(sh_pass(ctx, a));
    ShArgs b = base(Nv, 1, 0);  // DFT along dim 2, weighted |.|^2 (unitary: 1/(N1 N2))
    b.in = t;
    b.post = POST_TRACE_GRID;
    b.wgrid = wgrid;
    b.scale = 1.0f / ((float)N[0] * (float)N[1]);
    b.sum = sum;
    DIS_TRY(sh_pass(ctx, b));
  }
  return read_sum(ctx, sum, tr);
}

disorder_ctx_s* dis_shearlet_ctx(const disorder_shearlet_s* sh) { return sh->ctx; }
void dis_shearlet_size(const disorder_shearlet_s* sh, int* N) {
  for (int m = 0; m < 3; ++m) N[m] = sh->N[m];
}

namespace {

// probe[2e], probe[2e+1] = the two normals of (seed, e); sum += their squares
__global__ void probe_kernel(float* __restrict__ probe, long long V, uint64_t seed, double* __restrict__ sum) {
  __shared__ double red[kThr / 32];
  double part = 0.0;
  const long long n2 = (V + 1) / 2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n2; e += (long long)gridDim.x * blockDim.x) {
    float rad, c, s;
    dis_normal2_polar(seed, e, &rad, &c, &s);
    const float a = rad * c, b = rad * s;
    probe[2 * e] = a;
    part += (double)a * a;
    if (2 * e + 1 < V) {
      probe[2 * e + 1] = b;
      part += (double)b * b;
    }
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < kThr / 32; ++w) t += red[w];
    atomicAdd(sum, t);
  }
}

// probe *= (sum / V)^-1/2 (times the mask when given)
__global__ void probe_scale_kernel(float* __restrict__ probe, long long V, const double* __restrict__ sum,
                                   const float* __restrict__ mask) {
  const float s = (float)(1.0 / sqrt(*sum / (double)V));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < V; i += (long long)gridDim.x * blockDim.x)
    probe[i] = mask ? probe[i] * s * mask[i] : probe[i] * s;
}

}  // namespace

int disorder_trace_probe(disorder_ctx ctx, int64_t V, uint64_t seed, const float* mask, float* probe) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!probe || V < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "trace_probe: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  Workspace sw;
  DIS_TRY(dis_small(ctx, &sw));
  double* sum = sw.take<double>(1);
  DIS_CUDA_TRY(cudaMemsetAsync(sum, 0, sizeof(double), ctx->stream));
  const int blocks = (int)std::min<long long>(((V + 1) / 2 + kThr - 1) / kThr, 8LL * ctx->sm_count);
  probe_kernel<<<blocks, kThr, 0, ctx->stream>>>(probe, V, seed, sum);
  dis_count(ctx);
  const int b2 = (int)std::min<long long>((V + kThr - 1) / kThr, 8LL * ctx->sm_count);
  probe_scale_kernel<<<b2, kThr, 0, ctx->stream>>>(probe, V, sum, mask);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}
