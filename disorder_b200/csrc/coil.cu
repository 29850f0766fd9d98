// Coil stage of the encoding operators: coil expansion, the unitary 2-D DFT
// over the phase encodes, per-segment sample gather/scatter, k-space
// weighting, and the conj-coil combination (Reconstruction/encode.m:90-136,
// decode.m:42-58,78-85, encodedecode.m:91-178). The per-sample DFT rows of the
// reference (Fs{1}, Fs{2}: rows of build1DFTM(N,1)) are evaluated as a full
// FFT along dim 1 followed by an FFT along dim 2 and a gather of each
// segment's samples, which is the same linear map.
#include <cmath>

#include "fastpass.h"
#include "internal.h"

namespace {

constexpr int kThreads = 256;

struct Tile0 {  // axis-0 tile: L consecutive contiguous lines of an N1 x (N2*N3c) slab
  long long base[32];
  bool valid[32];
};

DIS_D void tile0(int N1, long long nlines, int L, int tile, Tile0* t, int tid) {
  if (tid < L) {
    long long q = (long long)tile * L + tid;
    t->valid[tid] = q < nlines;
    t->base[tid] = q < nlines ? q * N1 : 0;
  }
}

// load buf[p*P+l] = src[base[l] + p] (* mul[base[l]+p] when mul)
DIS_D void load0(const float2* __restrict__ src, float2* buf, const Tile0& t, int n, int L, int P,
                 int tid, int nthr) {
  for (int e = tid; e < n * L; e += nthr) {
    const int l = e / n, p = e - l * n;
    buf[p * P + l] = t.valid[l] ? src[t.base[l] + p] : make_float2(0.f, 0.f);
  }
}

__global__ void __launch_bounds__(kThreads) expand_fft1_kernel(CoilArgs a, const float2* __restrict__ z,
                                                               float2* __restrict__ A, int L, FFTPlan plan) {
  extern __shared__ float2 sm[];
  __shared__ Tile0 tl;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.N1, P = L + 1;
  float2* tw = sm;
  float2* bz = sm + ((n + 1) & ~1);
  float2* ba = bz + (long long)n * P;
  float2* bb = ba + (long long)n * P;
  const long long nlines = (long long)a.N2 * a.N3c;
  const long long Vc = nlines * n;
  load_twiddles(tw, n, tid, nthr);
  tile0(n, nlines, L, blockIdx.x, &tl, tid);
  __syncthreads();
  const int slot = blockIdx.y;
  load0(z + slot * a.Vz, bz, tl, n, L, P, tid, nthr);
  for (int c = 0; c < a.C; ++c) {
    const float2* S = a.Sf + c * a.Sc;
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e / n, p = e - l * n;
      float2 v = make_float2(0.f, 0.f);
      if (tl.valid[l]) v = cmul(S[tl.base[l] + p], bz[p * P + l]);
      ba[p * P + l] = v;
    }
    __syncthreads();
    float2* R = fft_tile(ba, bb, tw, plan, L, P, tid, nthr);
    float2* out = A + ((long long)slot * a.C + c) * Vc;
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e / n, p = e - l * n;
      if (tl.valid[l]) out[tl.base[l] + p] = R[p * P + l];
    }
    __syncthreads();
  }
}

// axis-1 tile over the slab of one (slot, coil): L consecutive ky rows at a
// fixed readout position n3; element (kz, l) at ky0 + l + kz*N1 + n3*N1*N2.
struct Tile1 {
  int ky0, n3, nl;
};

DIS_D Tile1 tile1(int N1, int L, int tile) {
  const int nt0 = (N1 + L - 1) / L;
  Tile1 t;
  t.n3 = tile / nt0;
  t.ky0 = (tile % nt0) * L;
  t.nl = min(L, N1 - t.ky0);
  return t;
}

__global__ void __launch_bounds__(kThreads) fft2_gather_kernel(CoilArgs a, const float2* __restrict__ A,
                                                              float2* __restrict__ y, long long ld, int n3off,
                                                              int N3y, const float2* __restrict__ ymeas,
                                                              float scale, int L, FFTPlan plan,
                                                              const int* __restrict__ rowptr,
                                                              const int* __restrict__ perm,
                                                              const int* __restrict__ kyv,
                                                              const int* __restrict__ kzv) {
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.N2, P = L + 1, N1 = a.N1;
  float2* tw = sm;
  float2* ba = sm + ((n + 1) & ~1);
  float2* bb = ba + (long long)n * P;
  load_twiddles(tw, n, tid, nthr);
  const Tile1 t = tile1(N1, L, blockIdx.x);
  const int c = blockIdx.y, slot = blockIdx.z;
  const long long Vc = (long long)N1 * a.N2 * a.N3c;
  const float2* src = A + ((long long)slot * a.C + c) * Vc + t.ky0 + (long long)t.n3 * N1 * a.N2;
  for (int e = tid; e < n * L; e += nthr) {
    const int p = e / L, l = e - p * L;
    ba[p * P + l] = l < t.nl ? src[l + (long long)p * N1] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* R = fft_tile(ba, bb, tw, plan, L, P, tid, nthr);
  const int seg = a.d_slot_seg[slot];
  const int* rp = rowptr + (long long)seg * (N1 + 1);
  const int s0 = rp[t.ky0], s1 = rp[t.ky0 + t.nl];
  const long long obase = ld * (t.n3 + n3off) + ld * N3y * c;
  for (int q = s0 + tid; q < s1; q += nthr) {
    const int i = perm[q];
    const int ky = kyv[i], kz = kzv[i];
    float2 v = cscale(R[kz * P + (ky - t.ky0)], scale);
    if (ymeas) v = csub(v, ymeas[obase + i]);
    y[obase + i] = v;
  }
}

__global__ void __launch_bounds__(kThreads) scatter_ifft2_kernel(CoilArgs a, const float2* __restrict__ y,
                                                                long long ld, int n3off, int N3y,
                                                                const float* __restrict__ We,
                                                                const float* __restrict__ Mb,
                                                                float2* __restrict__ A, int L, FFTPlan plan,
                                                                const int* __restrict__ rowptr,
                                                                const int* __restrict__ perm,
                                                                const int* __restrict__ kyv,
                                                                const int* __restrict__ kzv) {
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.N2, P = L + 1, N1 = a.N1;
  float2* tw = sm;
  float2* ba = sm + ((n + 1) & ~1);
  float2* bb = ba + (long long)n * P;
  load_twiddles(tw, n, tid, nthr);
  const Tile1 t = tile1(N1, L, blockIdx.x);
  const int c = blockIdx.y, slot = blockIdx.z;
  for (int e = tid; e < n * P; e += nthr) ba[e] = make_float2(0.f, 0.f);
  __syncthreads();
  const int seg = a.d_slot_seg[slot];
  const int* rp = rowptr + (long long)seg * (N1 + 1);
  const int s0 = rp[t.ky0], s1 = rp[t.ky0 + t.nl];
  const long long ibase = ld * (t.n3 + n3off) + ld * N3y * c;
  const float mb = Mb ? Mb[t.n3 + n3off] : 1.f;
  for (int q = s0 + tid; q < s1; q += nthr) {
    const int i = perm[q];
    const int ky = kyv[i], kz = kzv[i];
    float w = mb;
    if (We) w *= We[i];
    const float2 v = cscale(y[ibase + i], w);
    // conj(.) for the inverse via conj(FFT(conj(.)))
    atomicAdd(&ba[kz * P + (ky - t.ky0)].x, v.x);
    atomicAdd(&ba[kz * P + (ky - t.ky0)].y, -v.y);
  }
  __syncthreads();
  float2* R = fft_tile(ba, bb, tw, plan, L, P, tid, nthr);
  const long long Vc = (long long)N1 * a.N2 * a.N3c;
  float2* dst = A + ((long long)slot * a.C + c) * Vc + t.ky0 + (long long)t.n3 * N1 * a.N2;
  for (int e = tid; e < n * L; e += nthr) {
    const int p = e / L, l = e - p * L;
    if (l < t.nl) dst[l + (long long)p * N1] = cconj(R[p * P + l]);
  }
}

__global__ void __launch_bounds__(kThreads) fft2_weight_kernel(CoilArgs a, float2* __restrict__ A,
                                                              const float* __restrict__ wmap, int L,
                                                              FFTPlan plan) {
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.N2, P = L + 1, N1 = a.N1;
  float2* tw = sm;
  float2* ba = sm + ((n + 1) & ~1);
  float2* bb = ba + (long long)n * P;
  load_twiddles(tw, n, tid, nthr);
  const Tile1 t = tile1(N1, L, blockIdx.x);
  const int c = blockIdx.y, slot = blockIdx.z;
  const long long Vc = (long long)N1 * a.N2 * a.N3c;
  float2* src = A + ((long long)slot * a.C + c) * Vc + t.ky0 + (long long)t.n3 * N1 * a.N2;
  for (int e = tid; e < n * L; e += nthr) {
    const int p = e / L, l = e - p * L;
    ba[p * P + l] = l < t.nl ? src[l + (long long)p * N1] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* X = fft_tile(ba, bb, tw, plan, L, P, tid, nthr);
  float2* Xs = (X == ba) ? bb : ba;
  const int seg = a.d_slot_seg[slot];
  const float* wm = wmap + ((long long)seg * N1 + t.ky0) * a.N2;
  for (int e = tid; e < n * L; e += nthr) {
    const int p = e / L, l = e - p * L;
    const float w = l < t.nl ? wm[(long long)l * a.N2 + p] : 0.f;
    X[p * P + l] = cconj(cscale(X[p * P + l], w));
  }
  __syncthreads();
  float2* R = fft_tile(X, Xs, tw, plan, L, P, tid, nthr);
  for (int e = tid; e < n * L; e += nthr) {
    const int p = e / L, l = e - p * L;
    if (l < t.nl) src[l + (long long)p * N1] = cconj(R[p * P + l]);
  }
}

__global__ void __launch_bounds__(kThreads) ifft1_combine_kernel(CoilArgs a, const float2* __restrict__ A,
                                                                float2* __restrict__ u, float scale, int L,
                                                                FFTPlan plan) {
  extern __shared__ float2 sm[];
  __shared__ Tile0 tl;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = a.N1, P = L + 1;
  float2* tw = sm;
  float2* acc = sm + ((n + 1) & ~1);
  float2* ba = acc + (long long)n * P;
  float2* bb = ba + (long long)n * P;
  const long long nlines = (long long)a.N2 * a.N3c;
  const long long Vc = nlines * n;
  load_twiddles(tw, n, tid, nthr);
  tile0(n, nlines, L, blockIdx.x, &tl, tid);
  for (int e = tid; e < n * P; e += nthr) acc[e] = make_float2(0.f, 0.f);
  __syncthreads();
  const int slot = blockIdx.y;
  for (int c = 0; c < a.C; ++c) {
    const float2* src = A + ((long long)slot * a.C + c) * Vc;
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e / n, p = e - l * n;
      ba[p * P + l] = tl.valid[l] ? cconj(src[tl.base[l] + p]) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* R = fft_tile(ba, bb, tw, plan, L, P, tid, nthr);
    const float2* S = a.Sf + c * a.Sc;
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e / n, p = e - l * n;
      if (tl.valid[l]) {
        // conj(R) is the inverse DFT; times conj(S)
        const float2 v = cconj(R[p * P + l]);
        acc[p * P + l] = cadd(acc[p * P + l], cmulc(v, S[tl.base[l] + p]));
      }
    }
    __syncthreads();
  }
  float2* o = u + slot * a.Vz;
  for (int e = tid; e < n * L; e += nthr) {
    const int l = e / n, p = e - l * n;
    if (tl.valid[l]) o[tl.base[l] + p] = cscale(acc[p * P + l], scale);
  }
}

__global__ void weight_map_kernel(const int* __restrict__ segof, const int* __restrict__ kyv,
                                  const int* __restrict__ kzv, const float* __restrict__ We, long long ns,
                                  int N1, int N2, float* __restrict__ wmap, float scale, int n_seg,
                                  int* __restrict__ err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ns; i += (long long)gridDim.x * blockDim.x) {
    const float w = (We ? We[i] : 1.f) * scale;
    if (!DIS_DEBUG_INDEX(segof[i], n_seg, err, DIS_SITE_WEIGHT_MAP) || !DIS_DEBUG_INDEX(kyv[i], N1, err, DIS_SITE_WEIGHT_MAP) ||
        !DIS_DEBUG_INDEX(kzv[i], N2, err, DIS_SITE_WEIGHT_MAP))
      continue;
    atomicAdd(&wmap[((long long)segof[i] * N1 + kyv[i]) * N2 + kzv[i]], w);
  }
}

int pick_L(int n, int nbuf) {
  int L = 32;
  while (L > 2 && (size_t)nbuf * n * (L + 1) * sizeof(float2) > 100 * 1024) L >>= 1;
  return L;
}

template <class K>
void set_smem_attr(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

size_t smem_bytes(int n, int nbuf, int L) {
  return (size_t)((n + 1) & ~1) * sizeof(float2) + (size_t)nbuf * n * (L + 1) * sizeof(float2);
}

struct AttrInit {
  AttrInit() {
    set_smem_attr(expand_fft1_kernel);
    set_smem_attr(fft2_gather_kernel);
    set_smem_attr(scatter_ifft2_kernel);
    set_smem_attr(fft2_weight_kernel);
    set_smem_attr(ifft1_combine_kernel);
  }
};
void ensure_attrs() { static AttrInit once; }

}  // namespace

int dis_coil_expand_fft1(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* z,
                         float2* A) {
  if (a.n_slots == 0 || a.N3c == 0) return DISORDER_OK;
  if (dis_use_fast() && dis_fast_expand(a.N1, a, z, A, plan->d_tw[0], ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  ensure_attrs();
  const int n = a.N1;
  const int L = pick_L(n, 3);
  const long long nlines = (long long)a.N2 * a.N3c;
  dim3 grid((unsigned)((nlines + L - 1) / L), (unsigned)a.n_slots);
  if (!grid.x || !grid.y) return DISORDER_OK;
  expand_fft1_kernel<<<grid, kThreads, smem_bytes(n, 3, L), ctx->stream>>>(a, z, A, L, plan->fft[0]);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int dis_coil_fft2_gather(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* A,
                         float2* y, long long y_ld, int y_n3off, int y_N3, const float2* y_meas, float scale) {
  if (a.n_slots == 0 || a.N3c == 0) return DISORDER_OK;
  if (dis_use_fast() && dis_use_pipe() &&
      dis_fast_tma_gather(ctx, plan, a, A, y, y_ld, y_n3off, y_N3, y_meas, scale)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  if (dis_use_fast() && dis_fast_axis1(a.N2, 0, a, const_cast<float2*>(A), y, y_meas, y_ld, y_n3off, y_N3, scale,
                                       nullptr, nullptr, nullptr, plan, plan->d_tw[1], ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  ensure_attrs();
  const int n = a.N2;
  const int L = pick_L(n, 2);
  dim3 grid((unsigned)(((a.N1 + L - 1) / L) * a.N3c), (unsigned)a.C, (unsigned)a.n_slots);
  if (!grid.x || !grid.y || !grid.z) return DISORDER_OK;
  fft2_gather_kernel<<<grid, kThreads, smem_bytes(n, 2, L), ctx->stream>>>(
      a, A, y, y_ld, y_n3off, y_N3, y_meas, scale, L, plan->fft[1], plan->d_rowptr, plan->d_perm, plan->d_ky,
      plan->d_kz);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int dis_coil_scatter_ifft2(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* y,
                           long long y_ld, int y_n3off, int y_N3, const float* We, const float* Mb, float2* A) {
  if (a.n_slots == 0 || a.N3c == 0) return DISORDER_OK;
  if (dis_use_fast() && dis_use_pipe() && dis_fast_tma_scatter(ctx, plan, a, y, y_ld, y_n3off, y_N3, We, Mb, A)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  if (dis_use_fast() && dis_fast_axis1(a.N2, 2, a, A, const_cast<float2*>(y), nullptr, y_ld, y_n3off, y_N3, 1.f,
                                       nullptr, We, Mb, plan, plan->d_tw[1], ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  ensure_attrs();
  const int n = a.N2;
  const int L = pick_L(n, 2);
  dim3 grid((unsigned)(((a.N1 + L - 1) / L) * a.N3c), (unsigned)a.C, (unsigned)a.n_slots);
  if (!grid.x || !grid.y || !grid.z) return DISORDER_OK;
  scatter_ifft2_kernel<<<grid, kThreads, smem_bytes(n, 2, L), ctx->stream>>>(
      a, y, y_ld, y_n3off, y_N3, We, Mb, A, L, plan->fft[1], plan->d_rowptr, plan->d_perm, plan->d_ky, plan->d_kz);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int dis_coil_fft2_weight(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, float2* A,
                         const float* wmap, float2* ys, long long ys_ld, int ys_n3off, int ys_N3) {
  if (a.n_slots == 0 || a.N3c == 0) return DISORDER_OK;
  // the fast kernels apply w and the explicit inverse; the 1/(N1*N2) of the
  // inverse DFTs is applied by the combine step
  const float enc_scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
  if (dis_use_fast() && dis_use_pipe() &&
      dis_fast_tma_weight(ctx, a, A, wmap, plan->d_tw[1], plan, ys, ys_ld, ys_n3off, ys_N3, enc_scale)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  // the forward samples from a separate gather when the fused pass does not apply
  if (ys) DIS_TRY(dis_coil_fft2_gather(ctx, plan, a, A, ys, ys_ld, ys_n3off, ys_N3, nullptr, enc_scale));
  if (dis_use_fast() && dis_use_pipe() && dis_fast_wpipe(a.N2, a, A, wmap, plan->d_tw[1], ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  if (dis_use_fast() && dis_fast_axis1(a.N2, 1, a, A, nullptr, nullptr, 0, 0, 0, 1.f, wmap, nullptr, nullptr, plan,
                                       plan->d_tw[1], ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  ensure_attrs();
  const int n = a.N2;
  const int L = pick_L(n, 2);
  dim3 grid((unsigned)(((a.N1 + L - 1) / L) * a.N3c), (unsigned)a.C, (unsigned)a.n_slots);
  if (!grid.x || !grid.y || !grid.z) return DISORDER_OK;
  fft2_weight_kernel<<<grid, kThreads, smem_bytes(n, 2, L), ctx->stream>>>(a, A, wmap, L, plan->fft[1]);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int dis_coil_ifft1_combine(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* A,
                           float2* u, float scale) {
  if (a.n_slots == 0 || a.N3c == 0) return DISORDER_OK;
  if (dis_use_fast() && dis_fast_combine(a.N1, a, A, u, scale, plan->d_tw[0], ctx->stream)) {
    dis_count(ctx);
    DIS_CUDA_TRY(cudaGetLastError());
    return DISORDER_OK;
  }
  ensure_attrs();
  const int n = a.N1;
  const int L = pick_L(n, 3);
  const long long nlines = (long long)a.N2 * a.N3c;
  dim3 grid((unsigned)((nlines + L - 1) / L), (unsigned)a.n_slots);
  if (!grid.x || !grid.y) return DISORDER_OK;
  ifft1_combine_kernel<<<grid, kThreads, smem_bytes(n, 3, L), ctx->stream>>>(a, A, u, scale, L, plan->fft[0]);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int dis_build_weight_map(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float* We, float* wmap,
                         float scale) {
  const long long n = (long long)plan->n_seg * plan->N[0] * plan->N[1];
  DIS_CUDA_TRY(cudaMemsetAsync(wmap, 0, n * sizeof(float), ctx->stream));
  if (plan->n_samples == 0) return DISORDER_OK;
  const int blocks = (int)std::min<long long>((plan->n_samples + 255) / 256, 4096);
  weight_map_kernel<<<blocks, 256, 0, ctx->stream>>>(plan->d_seg_of, plan->d_ky, plan->d_kz, We, plan->n_samples,
                                                     plan->N[0], plan->N[1], wmap, scale, plan->n_seg, ctx->d_err);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

// ---------------------------------------------------------------- per-segment sums
// For every slot j (segment s = seg[j]) sums over the samples of s, the
// readout positions n3 < N3c and the coils:
//   out[j][0]      = sum |r|^2 * wrow[n3]
//   out[j][1+g]    = sum Re(G_g conj(r))              g < 6   (LMsolver.m:106)
//   out[j][7+h]    = sum Re(G_a conj(G_b)), (a,b)=ha_h h < 21 (LMsolver.m:115)
// Block partials are written per (slot, block) and reduced in a fixed order.
namespace {

__constant__ int c_ha[21][2];

constexpr int kSumBlocks = 64;

template <bool WITH_G>
__global__ void __launch_bounds__(256) seg_sums_kernel(const int* __restrict__ slot_seg,
                                                       const long long* __restrict__ seg_off,
                                                       const float2* __restrict__ r, const float2* __restrict__ G,
                                                       long long Gs, long long ld, int n3off, int N3c, int N3full,
                                                       int C, const float* __restrict__ wrow,
                                                       double* __restrict__ part) {
  const int slot = blockIdx.y;
  const int seg = slot_seg[slot];
  const long long i0 = seg_off[seg], i1 = seg_off[seg + 1];
  const long long ns = i1 - i0;
  const long long total = ns * (long long)N3c * C;
  constexpr int NT = WITH_G ? 28 : 1;
  double acc[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) acc[t] = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = i0 + e % ns;
    const long long rc = e / ns;
    const int n3 = (int)(rc % N3c) + n3off;
    const long long c = rc / N3c;
    const long long idx = i + ld * (n3 + (long long)N3full * c);
    const float2 rv = r[idx];
    const float wr = wrow ? wrow[n3] : 1.f;
    acc[0] += (double)wr * ((double)rv.x * rv.x + (double)rv.y * rv.y);
    if constexpr (WITH_G) {
      float2 g[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) g[q] = G[q * Gs + idx];
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[1 + q] += (double)g[q].x * rv.x + (double)g[q].y * rv.y;
#pragma unroll
      for (int h = 0; h < 21; ++h) {
        const float2 ga = g[c_ha[h][0]], gb = g[c_ha[h][1]];
        acc[7 + h] += (double)ga.x * gb.x + (double)ga.y * gb.y;
      }
    }
  }
  __shared__ double red[8][NT];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    double v = acc[t];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][t] = v;
  }
  __syncthreads();
  if (threadIdx.x < NT) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    part[((long long)slot * gridDim.x + blockIdx.x) * NT + threadIdx.x] = v;
  }
}

__global__ void seg_sums_final(const double* __restrict__ part, int nblk, int NT, int n_slots,
                               double* __restrict__ out) {
  const int j = blockIdx.x;
  for (int t = threadIdx.x; t < NT; t += blockDim.x) {
    double v = 0.0;
    for (int b = 0; b < nblk; ++b) v += part[((long long)j * nblk + b) * NT + t];
    out[(long long)j * 28 + t] = v;
  }
}

struct HaInit {
  HaInit() {
    int ha[21][2];
    int h = 0;
    for (int i = 0; i < 6; ++i) {
      ha[h][0] = i;
      ha[h][1] = i;
      ++h;
    }
    for (int i = 0; i < 6; ++i)
      for (int j = i + 1; j < 6; ++j) {
        ha[h][0] = i;
        ha[h][1] = j;
        ++h;
      }
    cudaMemcpyToSymbol(c_ha, ha, sizeof(ha));
  }
};

}  // namespace

int dis_seg_sums(disorder_ctx_s* ctx, const disorder_plan_s* plan, const int* d_slot_seg, int n_slots,
                 const float2* r, const float2* G, long long G_stride, long long ld, int n3off, int N3c, int N3full,
                 int C, const float* wrow, double* d_out, Workspace* ws) {
  static HaInit once;
  (void)once;
  if (n_slots == 0) return DISORDER_OK;
  const int NT = G ? 28 : 1;
  double* part = ws->take<double>((size_t)n_slots * kSumBlocks * NT);
  if (!part) return dis_set_error(ctx, DISORDER_OOM, "seg_sums: workspace too small");
  dim3 grid(kSumBlocks, n_slots);
  if (G)
    seg_sums_kernel<true><<<grid, 256, 0, ctx->stream>>>(d_slot_seg, plan->d_seg_off, r, G, G_stride, ld, n3off, N3c,
                                                          N3full, C, wrow, part);
  else
    seg_sums_kernel<false><<<grid, 256, 0, ctx->stream>>>(d_slot_seg, plan->d_seg_off, r, G, G_stride, ld, n3off, N3c,
                                                           N3full, C, wrow, part);
  seg_sums_final<<<n_slots, 32, 0, ctx->stream>>>(part, kSumBlocks, NT, n_slots, d_out);
  dis_count(ctx, 2);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}
