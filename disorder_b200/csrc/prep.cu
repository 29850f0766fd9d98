// Data preparation around the hot path on the device:
//  - Fourier resampling (Methods/resampling.m:45-94, image-space input, no
//    mirroring): per changed axis DFT/Nin, centred crop or zero-pad, inverse
//    DFT*Nout;
//  - sample gather for a pyramid level (the k-space crop of downsampleOperators,
//    Methods/downsampleOperators.m:48-51, applied to a sample list);
//  - coil compression (Methods/compressCoils.m:76-118): Gram matrix on the
//    device (double accumulation), Hermitian eigendecomposition on the host
//    (cyclic Jacobi), compression products on the device;
//  - the preconditioner A.Se = 1 ./ (sum_c |S_c|^2 + reg) (solveXT.m:231-233).
#include <algorithm>
#include <cmath>
#include <complex>
#include <numeric>
#include <vector>

#include "internal.h"

namespace {

constexpr int kThreads = 256;

struct ResampleArgs {
  int Din[3], Dout[3];
  int axis;
  int L, pitch;
  long long in_vs, out_vs;  // per-volume strides
  const float2* in;
  float2* out;
  FFTPlan pin, pout;
};

DIS_D int signed_freq(int j, int n) { return ((j + n / 2) % n) - n / 2; }

// one tile of L lines along `axis`: load Nin, FFT, map frequencies, inverse FFT of length Nout
__global__ void __launch_bounds__(kThreads) resample_kernel(ResampleArgs a) {
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int nin = a.pin.n, nout = a.pout.n, L = a.L, P = a.pitch;
  const int nmax = max(nin, nout);
  float2* twi = sm;
  float2* two = twi + ((nin + 1) & ~1);
  float2* b0 = two + ((nout + 1) & ~1);
  float2* b1 = b0 + (long long)nmax * P;
  float2* b2 = b1 + (long long)nmax * P;
  load_twiddles(twi, nin, tid, nthr);
  load_twiddles(two, nout, tid, nthr);
  // line enumeration over the other two axes (same for input and output)
  const int ax = a.axis;
  const int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;
  const long long nl = (long long)a.Din[o1] * a.Din[o2];
  const long long sin_ = ax == 0 ? 1 : (ax == 1 ? a.Din[0] : (long long)a.Din[0] * a.Din[1]);
  const long long sout = ax == 0 ? 1 : (ax == 1 ? a.Dout[0] : (long long)a.Dout[0] * a.Dout[1]);
  const int vol = blockIdx.y;
  const float2* in = a.in + vol * a.in_vs;
  float2* out = a.out + vol * a.out_vs;
  __syncthreads();
  for (int e = tid; e < nin * L; e += nthr) {
    const int l = e % L, p = e / L;
    const long long q = (long long)blockIdx.x * L + l;
    float2 v = make_float2(0.f, 0.f);
    if (q < nl) {
      const long long c1 = q % a.Din[o1], c2 = q / a.Din[o1];
      const long long base = ax == 0 ? (c1 + c2 * a.Din[1]) * a.Din[0]
                                     : (ax == 1 ? c1 + c2 * (long long)a.Din[0] * a.Din[1] : c1 + c2 * a.Din[0]);
      v = in[base + p * sin_];
    }
    b0[p * P + l] = v;
  }
  __syncthreads();
  float2* X = fft_tile(b0, b1, twi, a.pin, L, P, tid, nthr);
  // conj(spectrum mapped to nout) for the inverse via conj(FFT(conj))
  for (int e = tid; e < nout * L; e += nthr) {
    const int l = e % L, j = e / L;
    const int f = signed_freq(j, nout);
    const int lo = -(nin / 2), hi = (nin + 1) / 2 - 1;
    float2 v = make_float2(0.f, 0.f);
    if (f >= lo && f <= hi) {
      const int qi = (f % nin + nin) % nin;
      v = X[qi * P + l];
    }
    b2[j * P + l] = make_float2(v.x / nin, -v.y / nin);
  }
  __syncthreads();
  float2* Y = fft_tile(b2, (X == b0) ? b0 : b1, two, a.pout, L, P, tid, nthr);
  for (int e = tid; e < nout * L; e += nthr) {
    const int l = e % L, p = e / L;
    const long long q = (long long)blockIdx.x * L + l;
    if (q < nl) {
      const long long c1 = q % a.Din[o1], c2 = q / a.Din[o1];
      const long long base = ax == 0 ? (c1 + c2 * a.Dout[1]) * a.Dout[0]
                                     : (ax == 1 ? c1 + c2 * (long long)a.Dout[0] * a.Dout[1] : c1 + c2 * a.Dout[0]);
      out[base + p * sout] = cconj(Y[p * P + l]);
    }
  }
}

// the caller's indices are checked: one outside [0, ld_in) gives a zero row
// and the site in the error word, never an out-of-bounds read
__global__ void gather_rows_kernel(const float2* __restrict__ in, long long ld_in, const int* __restrict__ idx,
                                   long long n_out, long long rows, float scale, float2* __restrict__ out,
                                   int* __restrict__ err) {
  const long long tot = n_out * rows;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % n_out, r = e / n_out;
    const int k = idx[i];
    out[e] = dis_index_ok(k, ld_in, err, DIS_SITE_GATHER_ROWS) ? cscale(in[k + ld_in * r], scale)
                                                               : make_float2(0.f, 0.f);
  }
}

__global__ void precond_kernel(const float2* __restrict__ S, int C, long long V, float reg, float* __restrict__ out) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int c = 0; c < C; ++c) {
      const float2 a = S[c * V + v];
      s = fmaf(a.x, a.x, fmaf(a.y, a.y, s));
    }
    out[v] = 1.0f / (s + reg);
  }
}

// Gram P(c,c') = sum_v S_c conj(S_c') / (sum_c |S_c|^2 + reg); each thread owns
// pairs (c,c') = (p / C, p % C) for p = tid, tid+256, ...; voxels are staged
// in shared memory in chunks of kV.
constexpr int kV = 32;
__global__ void __launch_bounds__(kThreads) gram_kernel(const float2* __restrict__ S, int C, long long V, float reg,
                                                        double* __restrict__ part) {
  extern __shared__ float2 sv[];  // [kV][C] scaled, [kV][C] raw
  float2* sa = sv;
  float2* sb = sv + kV * C;
  const int tid = threadIdx.x;
  const int np = C * C;
  double acc[8][2];
  for (int k = 0; k < 8; ++k) acc[k][0] = acc[k][1] = 0.0;
  for (long long v0 = (long long)blockIdx.x * kV; v0 < V; v0 += (long long)gridDim.x * kV) {
    __syncthreads();
    for (int e = tid; e < kV * C; e += kThreads) {
      const int j = e / C, c = e % C;
      const long long v = v0 + j;
      sb[e] = v < V ? S[c * V + v] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    if (tid < kV) {
      float n = 0.f;
      for (int c = 0; c < C; ++c) n = fmaf(sb[tid * C + c].x, sb[tid * C + c].x, fmaf(sb[tid * C + c].y, sb[tid * C + c].y, n));
      const float inv = 1.0f / (n + reg);
      for (int c = 0; c < C; ++c) sa[tid * C + c] = cscale(sb[tid * C + c], inv);
    }
    __syncthreads();
    for (int k = 0; k < 8; ++k) {
      const int p = tid + k * kThreads;
      if (p >= np) break;
      const int c = p / C, d = p % C;
      float re = 0.f, im = 0.f;
      for (int j = 0; j < kV; ++j) {
        const float2 a = sa[j * C + c], b = sb[j * C + d];  // a * conj(b)
        re = fmaf(a.x, b.x, fmaf(a.y, b.y, re));
        im = fmaf(a.y, b.x, fmaf(-a.x, b.y, im));
      }
      acc[k][0] += re;
      acc[k][1] += im;
    }
  }
  for (int k = 0; k < 8; ++k) {
    const int p = tid + k * kThreads;
    if (p >= np) break;
    part[((long long)blockIdx.x * np + p) * 2] = acc[k][0];
    part[((long long)blockIdx.x * np + p) * 2 + 1] = acc[k][1];
  }
}

// out[v, j] = sum_c A[j, c] in[v, c]  (A: Cout x Cin, row-major, in constant-size shared copy)
__global__ void compress_kernel(const float2* __restrict__ in, long long V, int Cin, const float2* __restrict__ A,
                                int Cout, float2* __restrict__ out) {
  extern __shared__ float2 sA[];
  for (int e = threadIdx.x; e < Cin * Cout; e += blockDim.x) sA[e] = A[e];
  __syncthreads();
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < V; v += (long long)gridDim.x * blockDim.x) {
    float2 x[64];
    for (int c = 0; c < Cin; ++c) x[c] = in[c * V + v];
    for (int j = 0; j < Cout; ++j) {
      float2 acc = make_float2(0.f, 0.f);
      for (int c = 0; c < Cin; ++c) acc = cfma(sA[j * Cin + c], x[c], acc);
      out[j * V + v] = acc;
    }
  }
}

// Cyclic Jacobi eigendecomposition of a Hermitian matrix (column-major n x n).
// Returns eigenvalues (descending) and eigenvectors (columns).
void herm_eig(int n, std::vector<std::complex<double>> A, std::vector<double>* w,
              std::vector<std::complex<double>>* U) {
  using cd = std::complex<double>;
  auto at = [&](int i, int j) -> cd& { return A[i + (size_t)j * n]; };
  std::vector<cd> Vm((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Vm[i + (size_t)i * n] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += std::norm(at(p, q));
    if (off < 1e-30) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const cd apq = at(p, q);
        const double mag = std::abs(apq);
        if (mag < 1e-300) continue;
        const double app = at(p, p).real(), aqq = at(q, q).real();
        // rotation that zeroes A(p,q): phase e = apq/|apq|, angle from the 2x2 real problem
        const cd e = apq / mag;
        const double theta = 0.5 * std::atan2(2 * mag, aqq - app);
        const double c = std::cos(theta), s = std::sin(theta);
        // columns p,q: A' = A G, G = [c, s e; -s conj(e), c] acting on (p,q)
        for (int k = 0; k < n; ++k) {
          const cd akp = at(k, p), akq = at(k, q);
          at(k, p) = c * akp - s * std::conj(e) * akq;
          at(k, q) = s * e * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const cd apk = at(p, k), aqk = at(q, k);
          at(p, k) = c * apk - s * e * aqk;
          at(q, k) = s * std::conj(e) * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const cd vkp = Vm[k + (size_t)p * n], vkq = Vm[k + (size_t)q * n];
          Vm[k + (size_t)p * n] = c * vkp - s * std::conj(e) * vkq;
          Vm[k + (size_t)q * n] = s * e * vkp + c * vkq;
        }
      }
  }
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return at(a, a).real() > at(b, b).real(); });
  w->resize(n);
  U->assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    (*w)[j] = at(ord[j], ord[j]).real();
    for (int k = 0; k < n; ++k) (*U)[k + (size_t)j * n] = Vm[k + (size_t)ord[j] * n];
  }
}

}  // namespace

int dis_resample_axis(disorder_ctx_s* ctx, const float2* in, const int* Din, int axis, int nout, int nvol,
                      long long in_vs, long long out_vs, float2* out) {
  ResampleArgs a;
  for (int i = 0; i < 3; ++i) {
    a.Din[i] = Din[i];
    a.Dout[i] = Din[i];
  }
  a.Dout[axis] = nout;
  a.axis = axis;
  const int nin = Din[axis];
  if (!dis_make_fft_plan(nin, &a.pin) || !dis_make_fft_plan(nout, &a.pout))
    return dis_set_error(ctx, DISORDER_BAD_ARG, "resample: size %d or %d has an unsupported prime factor", nin, nout);
  const int nmax = std::max(nin, nout);
  int L = 16;
  while (L > 1 && 3 * (size_t)nmax * (L + 1) * sizeof(float2) > 96 * 1024) L >>= 1;
  a.L = L;
  a.pitch = L + 1;
  a.in = in;
  a.out = out;
  a.in_vs = in_vs;
  a.out_vs = out_vs;
  const size_t smem = sizeof(float2) * (((nin + 1) & ~1) + ((nout + 1) & ~1) + 3 * (size_t)nmax * a.pitch);
  // set once per process (thread-safe static initialisation)
  static const cudaError_t attr =
      cudaFuncSetAttribute(resample_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  (void)attr;
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
  const long long nl = (long long)Din[o1] * Din[o2];
  dim3 grid((unsigned)((nl + L - 1) / L), (unsigned)nvol);
  resample_kernel<<<grid, kThreads, smem, ctx->stream>>>(a);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

extern "C" {

int disorder_resample(disorder_ctx ctx, const void* x, const int32_t* Nin, int32_t n_vols, const int32_t* Nout,
                      void* out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!x || !Nin || !Nout || !out || n_vols < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "resample: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  int cur[3] = {Nin[0], Nin[1], Nin[2]};
  const long long vin = (long long)cur[0] * cur[1] * cur[2];
  const long long vout = (long long)Nout[0] * Nout[1] * Nout[2];
  int nchg = 0;
  for (int m = 0; m < 3; ++m) nchg += (cur[m] != Nout[m]);
  if (nchg == 0) {
    DIS_CUDA_TRY(cudaMemcpyAsync(out, x, sizeof(float2) * vin * n_vols, cudaMemcpyDeviceToDevice, ctx->stream));
    return DISORDER_OK;
  }
  // intermediate volumes (largest intermediate size) in the operator workspace
  long long vmax = std::max(vin, vout);
  {
    int d[3] = {cur[0], cur[1], cur[2]};
    for (int m = 0; m < 3; ++m) {
      d[m] = Nout[m];
      vmax = std::max(vmax, (long long)d[0] * d[1] * d[2]);
    }
  }
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, 2 * sizeof(float2) * vmax * n_vols + (1 << 20), &ws));
  float2* t0 = ws.take<float2>(vmax * n_vols);
  float2* t1 = ws.take<float2>(vmax * n_vols);
  const float2* src = (const float2*)x;
  int done = 0;
  for (int m = 0; m < 3; ++m) {
    if (cur[m] == Nout[m]) continue;
    ++done;
    float2* dst = (done == nchg) ? (float2*)out : (done % 2 ? t0 : t1);
    const long long vi = (long long)cur[0] * cur[1] * cur[2];
    int nd[3] = {cur[0], cur[1], cur[2]};
    nd[m] = Nout[m];
    const long long vo = (long long)nd[0] * nd[1] * nd[2];
    DIS_TRY(dis_resample_axis(ctx, src, cur, m, Nout[m], n_vols, vi, vo, dst));
    src = dst;
    cur[m] = Nout[m];
  }
  return DISORDER_OK;
}

int disorder_gather_samples(disorder_ctx ctx, const void* y_in, int64_t n_in, int64_t rows, const int32_t* idx,
                            int64_t n_out, float scale, void* y_out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!y_in || !idx || !y_out || n_in < 0 || n_out < 0 || rows < 0)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "gather_samples: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  if (n_out == 0 || rows == 0) return DISORDER_OK;
  const long long tot = n_out * rows;
  const int blocks = (int)std::min<long long>((tot + 255) / 256, 16LL * ctx->sm_count);
  gather_rows_kernel<<<blocks, 256, 0, ctx->stream>>>((const float2*)y_in, n_in, idx, n_out, rows, scale,
                                                      (float2*)y_out, ctx->d_err);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int disorder_precondition_weights(disorder_ctx ctx, const void* Sf, int32_t n_coils, int64_t V, float reg,
                                  float* out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!Sf || !out || n_coils < 1 || V < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "precondition: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  const int blocks = (int)std::min<long long>((V + 255) / 256, 16LL * ctx->sm_count);
  precond_kernel<<<blocks, 256, 0, ctx->stream>>>((const float2*)Sf, n_coils, V, reg, out);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int disorder_compress_coils(disorder_ctx ctx, const void* S, int32_t C_in, int64_t V, const void* y, int64_t n_y,
                            double perc, int32_t C_max, void* S_out, void* y_out, int32_t* C_out, double* D,
                            double* U) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!S || C_in < 1 || C_in > 64 || V < 1 || !S_out || !C_out || (y && !y_out))
    return dis_set_error(ctx, DISORDER_BAD_ARG, "compress_coils: bad arguments (1 <= C <= 64)");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  const int np = C_in * C_in;
  // partial Gram matrices (double complex) must fit the 16 MB scratch buffer
  const int nb = std::max(1, std::min(4 * ctx->sm_count, (int)((14u << 20) / ((size_t)np * 16))));
  Workspace ws;
  DIS_TRY(dis_small(ctx, &ws));
  double* part = ws.take<double>((size_t)nb * np * 2);
  float2* dA = ws.take<float2>((size_t)np);
  if (!part || !dA) return dis_set_error(ctx, DISORDER_OOM, "compress_coils workspace");
  if (np > 8 * kThreads) return dis_set_error(ctx, DISORDER_BAD_ARG, "compress_coils: too many coils");
  int nb_used = nb;
  if (ctx->precision != DISORDER_PRECISION_FP32) {
    // the contraction on the tensor cores, one CTA per SM
    nb_used = std::min(nb, ctx->sm_count);
    DIS_TRY(dis_gram_umma(ctx, (const float2*)S, C_in, V, 1e-9f, part, nb_used, ctx->precision));
  } else {
    gram_kernel<<<nb, kThreads, 2 * kV * C_in * sizeof(float2), ctx->stream>>>((const float2*)S, C_in, V, 1e-9f,
                                                                              part);
    dis_count(ctx);
  }
  std::vector<double> h((size_t)nb_used * np * 2);
  DIS_CUDA_TRY(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->precision != DISORDER_PRECISION_FP32) {
    int late = 0;
    DIS_CUDA_TRY(cudaMemcpy(&late, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (late) {
      DIS_CUDA_TRY(cudaMemset(ctx->d_err, 0, sizeof(int)));
      return dis_set_error(ctx, DISORDER_TIMEOUT, "compress_coils: a tensor-core MMA wait ran out");
    }
  }
  std::vector<std::complex<double>> P((size_t)np, 0.0);
  for (int b = 0; b < nb_used; ++b)
    for (int p = 0; p < np; ++p) P[p] += std::complex<double>(h[((size_t)b * np + p) * 2], h[((size_t)b * np + p) * 2 + 1]);
  // P(c,d) with p = c*C + d -> column-major matrix M(c,d)
  std::vector<std::complex<double>> M((size_t)np);
  for (int c = 0; c < C_in; ++c)
    for (int d = 0; d < C_in; ++d) M[c + (size_t)d * C_in] = P[(size_t)c * C_in + d];
  std::vector<double> w;
  std::vector<std::complex<double>> Uv;
  herm_eig(C_in, M, &w, &Uv);
  for (auto& v : w) v = std::fabs(v);
  int Ck = C_in;
  if (perc < 1) {
    double tot = 0, cs = 0;
    for (double v : w) tot += v;
    Ck = C_in;
    for (int j = 0; j < C_in; ++j) {
      cs += w[j];
      if (cs / tot >= perc) {
        Ck = j + 1;
        break;
      }
    }
  } else {
    Ck = std::min<int>((int)perc, C_in);
  }
  if (C_max > 0) Ck = std::min(Ck, (int)C_max);
  *C_out = Ck;
  if (D)
    for (int j = 0; j < C_in; ++j) D[j] = w[j];
  if (U)
    for (size_t k = 0; k < Uv.size(); ++k) {
      U[2 * k] = Uv[k].real();
      U[2 * k + 1] = Uv[k].imag();
    }
  // A = U(:,1:Ck)^H, row-major Ck x C_in
  std::vector<float2> A((size_t)Ck * C_in);
  for (int j = 0; j < Ck; ++j)
    for (int c = 0; c < C_in; ++c) {
      const std::complex<double> u = std::conj(Uv[c + (size_t)j * C_in]);
      A[(size_t)j * C_in + c] = make_float2((float)u.real(), (float)u.imag());
    }
  DIS_CUDA_TRY(cudaMemcpyAsync(dA, A.data(), A.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
  const int blocks = (int)std::min<long long>((V + 255) / 256, 8LL * ctx->sm_count);
  compress_kernel<<<blocks, 256, A.size() * sizeof(float2), ctx->stream>>>((const float2*)S, V, C_in, dA, Ck,
                                                                           (float2*)S_out);
  dis_count(ctx);
  if (y) {
    const int yb = (int)std::min<long long>((n_y + 255) / 256, 8LL * ctx->sm_count);
    compress_kernel<<<yb, 256, A.size() * sizeof(float2), ctx->stream>>>((const float2*)y, n_y, C_in, dA, Ck,
                                                                         (float2*)y_out);
    dis_count(ctx);
  }
  DIS_CUDA_TRY(cudaGetLastError());
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

}  // extern "C"
