// CGsolver (Reconstruction/CGsolver.m) and LMsolver (Reconstruction/LMsolver.m).
// Vectors are single precision; every inner product and norm is accumulated
// in double precision with a deterministic two-stage reduction; the CG
// scalars and the LM 6x6 systems are double precision.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "encoding.h"
#include "internal.h"
#include "solvers.h"

namespace {

constexpr int kRedBlocks = 592;  // 4 x 148 SMs

struct d2 {
  double x, y;
};

DIS_D void block_reduce_d2(double& a, double& b, d2* out) {
  __shared__ double sa[32], sb[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    sa[wid] = a;
    sb[wid] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tb = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      ta += sa[w];
      tb += sb[w];
    }
    out->x = ta;
    out->y = tb;
  }
}

__global__ void final_reduce_kernel(const d2* __restrict__ part, int n, d2* __restrict__ res) {
  double a = 0, b = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    a += part[i].x;
    b += part[i].y;
  }
  __shared__ double sa[256], sb[256];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sa[threadIdx.x] += sa[threadIdx.x + s];
      sb[threadIdx.x] += sb[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    res->x = sa[0];
    res->y = sb[0];
  }
}

// sum conj(a) * b
__global__ void dot_kernel(const float2* __restrict__ a, const float2* __restrict__ b, long long n,
                           d2* __restrict__ part) {
  double re = 0, im = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 u = a[i], v = b[i];
    re += (double)u.x * v.x + (double)u.y * v.y;
    im += (double)u.x * v.y - (double)u.y * v.x;
  }
  block_reduce_d2(re, im, part + blockIdx.x);
}

// EHE = Ma .* (EHE + Ti .* p); partial sum conj(p) * EHE   (CGsolver.m:80,82)
__global__ void pap_kernel(const float2* __restrict__ p, float2* __restrict__ ehe, const float* __restrict__ Ma,
                           const float* __restrict__ Ti, long long n, d2* __restrict__ part) {
  double re = 0, im = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 pv = p[i];
    float2 e = ehe[i];
    if (Ti) e = cadd(e, cscale(pv, Ti[i]));
    if (Ma) e = cscale(e, Ma[i]);
    ehe[i] = e;
    re += (double)pv.x * e.x + (double)pv.y * e.y;
    im += (double)pv.x * e.y - (double)pv.y * e.x;
  }
  block_reduce_d2(re, im, part + blockIdx.x);
}

// x += g p; r -= g EHE; z = Se r; partial sum conj(z) r   (CGsolver.m:83-94)
__global__ void update_kernel(float2* __restrict__ x, float2* __restrict__ r, float2* __restrict__ z,
                              const float2* __restrict__ p, const float2* __restrict__ ehe, const float* __restrict__ Se,
                              float2 g, long long n, d2* __restrict__ part) {
  double re = 0, im = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 pv = p[i];
    x[i] = cadd(x[i], cmul(g, pv));
    const float2 rv = csub(r[i], cmul(g, ehe[i]));
    r[i] = rv;
    const float2 zv = Se ? cscale(rv, Se[i]) : rv;
    z[i] = zv;
    re += (double)zv.x * rv.x + (double)zv.y * rv.y;
    im += (double)zv.x * rv.y - (double)zv.y * rv.x;
  }
  block_reduce_d2(re, im, part + blockIdx.x);
}

// r = b - EHE; z = Se r; p = z; partial sum conj(z) r   (CGsolver.m:64-68)
__global__ void init_kernel(const float2* __restrict__ b, const float2* __restrict__ ehe, float2* __restrict__ r,
                            float2* __restrict__ z, float2* __restrict__ p, const float* __restrict__ Se, long long n,
                            d2* __restrict__ part) {
  double re = 0, im = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 rv = ehe ? csub(b[i], ehe[i]) : b[i];
    r[i] = rv;
    const float2 zv = Se ? cscale(rv, Se[i]) : rv;
    z[i] = zv;
    p[i] = zv;
    re += (double)zv.x * rv.x + (double)zv.y * rv.y;
    im += (double)zv.x * rv.y - (double)zv.y * rv.x;
  }
  block_reduce_d2(re, im, part + blockIdx.x);
}

// p = z + d p
// r = -y (the residual of x = 0)
__global__ void neg_kernel(float2* __restrict__ r, const float2* __restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = y[i];
    r[i] = make_float2(-v.x, -v.y);
  }
}

// r += g e (the sample residual follows x += g p with e = E p)
__global__ void caxpy_kernel(float2* __restrict__ r, const float2* __restrict__ e, float2 g, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    r[i] = cadd(r[i], cmul(g, e[i]));
}

__global__ void pupdate_kernel(float2* __restrict__ p, const float2* __restrict__ z, float2 d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = cadd(z[i], cmul(d, p[i]));
}

// sum |conj(Se b) b| (CGsolver.m:59-61) and sum Ti |x|^2 (computeEnergy.m:72-75)
__global__ void wnorm_kernel(const float2* __restrict__ b, const float* __restrict__ w, long long n,
                             d2* __restrict__ part) {
  double re = 0, im = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = b[i];
    const double q = (double)v.x * v.x + (double)v.y * v.y;
    re += (w ? (double)fabsf(w[i]) : 1.0) * q;
  }
  block_reduce_d2(re, im, part + blockIdx.x);
}

__global__ void constrain_kernel(float2* __restrict__ v, const float* __restrict__ Ma, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = cscale(v[i], Ma[i]);
}

__global__ void rowweight_kernel(const float* __restrict__ a, const float* __restrict__ b, int n, float* __restrict__ o) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) o[i] = (a ? a[i] : 1.f) * (b ? b[i] : 1.f);
}

}  // namespace

// ---------------------------------------------------------------- reductions
struct Reducer {
  disorder_ctx_s* ctx;
  d2* part;
  d2* res;
  d2* host;  // pinned
};

static int red_finish(Reducer& R, double* re, double* im) {
  disorder_ctx_s* ctx = R.ctx;
  final_reduce_kernel<<<1, 256, 0, ctx->stream>>>(R.part, kRedBlocks, R.res);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaMemcpyAsync(R.host, R.res, sizeof(d2), cudaMemcpyDeviceToHost, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  *re = R.host->x;
  if (im) *im = R.host->y;
  return DISORDER_OK;
}

static int red_init(disorder_ctx_s* ctx, Workspace* ws, Reducer* R) {
  R->ctx = ctx;
  R->part = ws->take<d2>(kRedBlocks);
  R->res = ws->take<d2>(1);
  if (!R->part || !R->res) return dis_set_error(ctx, DISORDER_OOM, "reduction workspace");
  if (!ctx->h_scalars) DIS_CUDA_TRY(cudaMallocHost(&ctx->h_scalars, sizeof(d2) * 4));
  R->host = static_cast<d2*>(ctx->h_scalars);
  return DISORDER_OK;
}

int dis_weighted_norm(disorder_ctx_s* ctx, const float2* b, const float* w, long long n, double* out) {
  Workspace ws;
  DIS_TRY(dis_small(ctx, &ws));
  Reducer R;
  DIS_TRY(red_init(ctx, &ws, &R));
  wnorm_kernel<<<kRedBlocks, 256, 0, ctx->stream>>>(b, w, n, R.part);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return red_finish(R, out, nullptr);
}

// ---------------------------------------------------------------- energy
// computeEnergy (Reconstruction/computeEnergy.m:34-80) for no=2.
int dis_energy(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* y, const float2* x, const float2* Sf,
               int C, const float* T, const float* rowW, const float* R_Ti, float2* rbuf, double* En, int n3_lo,
               int n3_cnt) {
  // readout rows outside [n3_lo, n3_lo + n3_cnt) have zero weight: their
  // samples are neither encoded nor summed (n3_cnt < 0: all rows)
  if (n3_cnt < 0 || !rowW) {
    n3_lo = 0;
    n3_cnt = plan->N[2];
  }
  double reg = 0;
  if (R_Ti) DIS_TRY(dis_ti_energy(ctx, x, R_Ti, plan->V, &reg));
  En[1] = reg;
  if (n3_cnt == 0) {
    En[0] = 0;
    return DISORDER_OK;
  }
  EncodeSpec sp;
  sp.x = x;
  sp.Sf = Sf;
  sp.C = C;
  sp.T = T;
  sp.T_n = plan->n_mot;
  for (int s = 0; s < plan->n_seg; ++s) sp.segs.push_back(s);
  sp.n3_lo = n3_lo;
  sp.N3c = n3_cnt;
  sp.y_ld = plan->n_samples;
  sp.y_n3off = n3_lo;
  sp.y_N3 = plan->N[2];
  DIS_TRY(dis_encode_segments(ctx, plan, sp, rbuf, y));
  return dis_fidelity(ctx, plan, rbuf, C, rowW, En, n3_lo, n3_cnt);
}

// En[0] = sum over the samples of rows [n3_lo, n3_lo + n3_cnt) of rowW[n3] |r|^2
// (all rows and weight 1 without rowW), for a residual r = E x - y in
// encode's layout.
int dis_fidelity(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* rbuf, int C, const float* rowW,
                 double* En, int n3_lo, int n3_cnt) {
  if (n3_cnt < 0 || !rowW) {
    n3_lo = 0;
    n3_cnt = plan->N[2];
  }
  if (n3_cnt == 0) {
    En[0] = 0;
    return DISORDER_OK;
  }
  // sum |r|^2 * rowW[n3] over all samples
  const long long n = plan->n_samples * plan->N[2] * (long long)C;
  Workspace ws;
  DIS_TRY(dis_small(ctx, &ws));
  Reducer R;
  DIS_TRY(red_init(ctx, &ws, &R));
  double fid = 0;
  if (!rowW) {
    wnorm_kernel<<<kRedBlocks, 256, 0, ctx->stream>>>(rbuf, nullptr, n, R.part);
    dis_count(ctx);
    DIS_TRY(red_finish(R, &fid, nullptr));
  } else {
    std::vector<int> all;
    for (int s = 0; s < plan->n_seg; ++s) all.push_back(s);
    int* d_all = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &ws, all, &d_all));
    double* d_out = ws.take<double>((size_t)plan->n_seg * 28);
    if (!d_out) return dis_set_error(ctx, DISORDER_OOM, "energy workspace");
    DIS_TRY(dis_seg_sums(ctx, plan, d_all, plan->n_seg, rbuf, nullptr, 0, plan->n_samples, n3_lo, n3_cnt,
                         plan->N[2], C, rowW, d_out, &ws));
    std::vector<double> h((size_t)plan->n_seg * 28);
    DIS_CUDA_TRY(cudaMemcpyAsync(h.data(), d_out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int s = 0; s < plan->n_seg; ++s) fid += h[(size_t)s * 28];
  }
  En[0] = fid;
  return DISORDER_OK;
}

namespace {
__global__ void ti_kernel(const float2* __restrict__ x, const float* __restrict__ ti, long long n, d2* __restrict__ part) {
  double re = 0, im = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = x[i];
    re += (double)ti[i] * ((double)v.x * v.x + (double)v.y * v.y);
  }
  block_reduce_d2(re, im, part + blockIdx.x);
}
}  // namespace

int dis_ti_energy(disorder_ctx_s* ctx, const float2* x, const float* ti, long long n, double* out) {
  Workspace ws;
  DIS_TRY(dis_small(ctx, &ws));
  Reducer R;
  DIS_TRY(red_init(ctx, &ws, &R));
  ti_kernel<<<kRedBlocks, 256, 0, ctx->stream>>>(x, ti, n, R.part);
  dis_count(ctx);
  double v = 0;
  DIS_TRY(red_finish(R, &v, nullptr));
  *out = std::fabs(v);
  return DISORDER_OK;
}

// ---------------------------------------------------------------- CG
int dis_cg_solve(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CGSpec& s, float2* x, int x_init, int nIt,
                 int tolType, double tol, double* En, int* n_en, int* nn) {
  const long long V = plan->V;
  const int NitTest = 2;  // CGsolver.m:37
  if (tolType != 1 && tolType != 6 && tolType != 7)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "CG: tolType %d not supported (1, 6 or 7)", tolType);
  // persistent solver vectors: b, r, z, p, ehe + wmap + residual buffer + row weights
  const long long wm = (long long)plan->n_seg * plan->N[0] * plan->N[1];
  const long long ny = plan->n_samples * plan->N[2] * (long long)s.C;
  // With the Energy tolerance the residual r = E x - y is kept in sample
  // space: each normal operator on p also writes E p (ebuf), r += g E p
  // follows x += g p, and the energy is a reduction of r, the same quantity
  // the reference gets from an encode of x (computeEnergy.m:52-70). The
  // plane path does not produce E p: it encodes x at each evaluation.
  std::vector<int> all_segs;
  for (int q = 0; q < plan->n_seg; ++q) all_segs.push_back(q);
  const bool track = (tolType == 6 || s.r_out) && !dis_plane_usable(plan, s.C, all_segs);
  // From an initial guess x0, with r = E x0 - y and without EH.Mb (which
  // decode applies and encodedecode does not), b - EHE(x0) =
  // -constrain(decode(W r) + Ti x0): one encode and one decode replace the
  // decode of y and the normal operator on x0 (:46, :53-56). b itself is
  // needed only by the RelativeResidual2Error test with a positive tolerance.
  const bool need_b = tolType == 1 && tol > 0;
  const bool fused_init = x_init && !s.Mb && (track || !need_b);
  const bool have_rbuf = tolType == 6 || fused_init || s.r_out;
  const size_t need = sizeof(float2) * (5 * V + (have_rbuf ? ny : 0) + (track ? ny : 0)) +
                      sizeof(float) * (wm + plan->N[2]) + (1 << 20);
  Workspace ws;
  DIS_TRY(dis_workspace2(ctx, need, &ws));
  float2* b = ws.take<float2>(V);
  float2* r = ws.take<float2>(V);
  float2* z = ws.take<float2>(V);
  float2* p = ws.take<float2>(V);
  float2* ehe = ws.take<float2>(V);
  float* wmap = ws.take<float>(wm);
  float* roww = ws.take<float>(plan->N[2]);
  float2* rbuf = have_rbuf ? ws.take<float2>(ny) : nullptr;
  float2* ebuf = track ? ws.take<float2>(ny) : nullptr;
  if (!b || !r || !z || !p || !ehe || !wmap || !roww || (have_rbuf && !rbuf) || (track && !ebuf))
    return dis_set_error(ctx, DISORDER_OOM, "CG workspace");
  DIS_TRY(dis_build_weight_map(ctx, plan, s.We, wmap, 1.f));
  const bool haveRow = s.Mb || s.Mbe;
  int e_lo = 0, e_cnt = -1;  // readout rows with nonzero energy weight
  if (haveRow) {
    rowweight_kernel<<<1, 256, 0, ctx->stream>>>(s.Mb, s.Mbe, plan->N[2], roww);
    dis_count(ctx);
    if (tolType == 6) {
      std::vector<float> hw(plan->N[2]);
      DIS_CUDA_TRY(cudaMemcpyAsync(hw.data(), roww, hw.size() * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
      DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      int lo = plan->N[2], hi = -1;
      for (int k = 0; k < plan->N[2]; ++k)
        if (hw[k] != 0.f) {
          lo = std::min(lo, k);
          hi = k;
        }
      e_lo = hi < 0 ? 0 : lo;
      e_cnt = hi < 0 ? 0 : hi - lo + 1;
    }
  }
  Workspace rws;
  DIS_TRY(dis_small(ctx, &rws));
  Reducer R;
  DIS_TRY(red_init(ctx, &rws, &R));
  std::vector<int> segs;
  for (int q = 0; q < plan->n_seg; ++q) segs.push_back(q);
  auto encode_residual = [&]() -> int {  // rbuf = E x - y
    EncodeSpec sp;
    sp.x = x;
    sp.Sf = s.Sf;
    sp.C = s.C;
    sp.T = s.T;
    sp.T_n = plan->n_mot;
    sp.segs = all_segs;
    sp.n3_lo = 0;
    sp.N3c = plan->N[2];
    sp.y_ld = plan->n_samples;
    sp.y_n3off = 0;
    sp.y_N3 = plan->N[2];
    return dis_encode_segments(ctx, plan, sp, rbuf, s.y);
  };
  // the final sample residual for the caller: the tracked one, else a fresh encode
  auto write_residual = [&](bool tracked) -> int {
    if (!s.r_out) return DISORDER_OK;
    if (!tracked) DIS_TRY(encode_residual());
    DIS_CUDA_TRY(cudaMemcpyAsync(s.r_out, rbuf, sizeof(float2) * ny, cudaMemcpyDeviceToDevice, ctx->stream));
    return DISORDER_OK;
  };
  // b = constrain(decode(y))   (:46)
  DecodeSpec ds;
  ds.y = s.y;
  ds.Sf = s.Sf;
  ds.C = s.C;
  ds.T = s.T;
  ds.T_n = plan->n_mot;
  ds.segs = segs;
  ds.We = s.We;
  ds.Mb = s.Mb;
  const int blocks = kRedBlocks;
  if (fused_init) {
    DIS_TRY(encode_residual());
    ds.y = rbuf;
    DIS_TRY(dis_decode_segments(ctx, plan, ds, ehe));  // E^H W (E x0 - y)
    DIS_CUDA_TRY(cudaMemsetAsync(b, 0, sizeof(float2) * V, ctx->stream));
  } else {
    DIS_TRY(dis_decode_segments(ctx, plan, ds, b));
    if (s.C_Ma) {
      constrain_kernel<<<blocks, 256, 0, ctx->stream>>>(b, s.C_Ma, V);
      dis_count(ctx);
    }
  }
  EncodeDecodeSpec es;
  es.x = nullptr;
  es.Sf = s.Sf;
  es.C = s.C;
  es.T = s.T;
  es.T_n = plan->n_mot;
  es.segs = segs;
  es.wmap = wmap;
  es.We = s.We;
  auto normal_op = [&](const float2* in, float2* out, float2* samples) -> int {
    es.x = in;
    es.ys = samples;
    return dis_encodedecode_segments(ctx, plan, es, out);
  };
  double dummy = 0;
  // EHE for the initial guess (:53-56)
  if (x_init) {
    if (!fused_init) DIS_TRY(normal_op(x, ehe, nullptr));
    if (s.sh) DIS_TRY(dis_shearlet_regularize(ctx, s.sh, x, s.sh_We, s.sh_scale, 1.f, ehe));
    pap_kernel<<<blocks, 256, 0, ctx->stream>>>(x, ehe, s.C_Ma, s.R_Ti, V, R.part);
    dis_count(ctx);
    DIS_TRY(red_finish(R, &dummy, nullptr));
  } else {
    DIS_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(float2) * V, ctx->stream));
  }
  double bnorm2 = 1.0;
  if (tolType != 6 && tolType != 7 && !fused_init) {  // :58-62 (unused when the tolerance is not positive)
    wnorm_kernel<<<blocks, 256, 0, ctx->stream>>>(b, s.P_Se, V, R.part);
    dis_count(ctx);
    DIS_TRY(red_finish(R, &bnorm2, nullptr));
  }
  init_kernel<<<blocks, 256, 0, ctx->stream>>>(b, x_init ? ehe : nullptr, r, z, p, s.P_Se, V, R.part);
  dis_count(ctx);
  double rs_re = 0, rs_im = 0;
  DIS_TRY(red_finish(R, &rs_re, &rs_im));
  *n_en = 0;
  *nn = 0;
  if (!std::isfinite(rs_re) || !std::isfinite(rs_im))
    return dis_set_error(ctx, DISORDER_NONFINITE, "CG: non-finite initial residual (non-finite y, x0 or weights)");
  if (std::hypot(rs_re, rs_im) < 1e-6) return write_residual(fused_init);  // :70-75
  if (track) {
    // r = E x0 - y (x0 = 0: r = -y)
    if (x_init) {
      if (!fused_init) DIS_TRY(encode_residual());
    } else {
      neg_kernel<<<blocks, 256, 0, ctx->stream>>>(rbuf, s.y, ny);
      dis_count(ctx);
    }
  }
  double err = INFINITY;
  std::vector<double> Ecol;  // energies of odd iterations, 2 per column
  int n = 0;
  for (n = 1; n <= nIt; ++n) {
    DIS_TRY(normal_op(p, ehe, ebuf));  // :80 (and E p for the residual)
    if (s.sh) DIS_TRY(dis_shearlet_regularize(ctx, s.sh, p, s.sh_We, s.sh_scale, 1.f, ehe));  // regularize.m:27-46
    pap_kernel<<<blocks, 256, 0, ctx->stream>>>(p, ehe, s.C_Ma, s.R_Ti, V, R.part);
    dis_count(ctx);
    double pa_re = 0, pa_im = 0;
    DIS_TRY(red_finish(R, &pa_re, &pa_im));
    if (!std::isfinite(pa_re) || !std::isfinite(pa_im))
      return dis_set_error(ctx, DISORDER_NONFINITE, "CG: non-finite <p, EHE p> at iteration %d", n);
    // g = rsold / <p, EHE>  (:82)
    const double den = pa_re * pa_re + pa_im * pa_im;
    const double g_re = (rs_re * pa_re + rs_im * pa_im) / den;
    const double g_im = (rs_im * pa_re - rs_re * pa_im) / den;
    // x += g p (:83-84); energy of odd iterations uses the updated x (:86-89)
    // r -= g EHE, z = P r, rs = <z, r>  (:90-94)  -- fused, x updated in the same pass
    update_kernel<<<blocks, 256, 0, ctx->stream>>>(x, r, z, p, ehe, s.P_Se, make_float2((float)g_re, (float)g_im), V,
                                                   R.part);
    dis_count(ctx);
    double rn_re = 0, rn_im = 0;
    DIS_TRY(red_finish(R, &rn_re, &rn_im));
    if (!std::isfinite(rn_re) || !std::isfinite(rn_im))
      return dis_set_error(ctx, DISORDER_NONFINITE, "CG: non-finite residual at iteration %d", n);
    if (track) {
      caxpy_kernel<<<blocks, 256, 0, ctx->stream>>>(rbuf, ebuf, make_float2((float)g_re, (float)g_im), ny);
      dis_count(ctx);
    }
    if (n % NitTest == 1 && tolType == 6) {
      double e2[2];
      if (track) {
        DIS_TRY(dis_fidelity(ctx, plan, rbuf, s.C, haveRow ? roww : nullptr, e2, e_lo, e_cnt));
        e2[1] = 0;
        if (s.R_Ti) DIS_TRY(dis_ti_energy(ctx, x, s.R_Ti, V, &e2[1]));
      } else {
        DIS_TRY(dis_energy(ctx, plan, s.y, x, s.Sf, s.C, s.T, haveRow ? roww : nullptr, s.R_Ti, rbuf, e2, e_lo,
                           e_cnt));
      }
      Ecol.push_back(e2[0]);
      Ecol.push_back(e2[1]);
    }
    // d = rs/(rsold+eps), p = z + d p  (:95-97)
    const double dr = rs_re + DBL_EPSILON, di = rs_im;
    const double dd = dr * dr + di * di;
    const double d_re = (rn_re * dr + rn_im * di) / dd;
    const double d_im = (rn_im * dr - rn_re * di) / dd;
    pupdate_kernel<<<blocks, 256, 0, ctx->stream>>>(p, z, make_float2((float)d_re, (float)d_im), V);
    dis_count(ctx);
    rs_re = rn_re;
    rs_im = rn_im;
    if (tolType == 1) {
      err = std::sqrt(std::hypot(rs_re, rs_im) / bnorm2);  // sum|conj(z) r| = sum Se|r|^2 for Se>=0
    } else if (tolType == 6 && n % NitTest == 1 && n > 1) {
      const size_t k = Ecol.size() / 2 - 1;
      const double prev = Ecol[2 * (k - 1)] + Ecol[2 * (k - 1) + 1];
      const double cur = Ecol[2 * k] + Ecol[2 * k + 1];
      err = (prev - cur) / prev;  // :100
    }
    if (err < tol || std::hypot(rs_re, rs_im) < 1e-6) break;  // :103
  }
  *nn = std::min(n, nIt);
  const int ncol = (int)(Ecol.size() / 2);
  if (En)
    for (int k = 0; k < ncol; ++k) {
      En[2 * k] = Ecol[2 * k];
      En[2 * k + 1] = Ecol[2 * k + 1];
    }
  *n_en = ncol;
  DIS_TRY(write_residual(track));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

// ---------------------------------------------------------------- LM
namespace {

// Hessian index pairs ha (LMsolver.m:26): the 6 diagonal entries, then nchoosek(1:6,2)
void ha_pairs(int ha[21][2]) {
  int h = 0;
  for (int i = 0; i < 6; ++i) {
    ha[h][0] = ha[h][1] = i;
    ++h;
  }
  for (int i = 0; i < 6; ++i)
    for (int j = i + 1; j < 6; ++j) {
      ha[h][0] = i;
      ha[h][1] = j;
      ++h;
    }
}

// double(MH)\g as MATLAB's mldivide does for a symmetric matrix with a
// positive diagonal: Cholesky, falling back to LU with partial pivoting.
void solve6(const double M[6][6], const double g[6], double x[6]) {
  double L[6][6] = {{0}};
  bool ok = true;
  for (int j = 0; j < 6 && ok; ++j) {
    double s = M[j][j];
    for (int k = 0; k < j; ++k) s -= L[j][k] * L[j][k];
    if (!(s > 0)) {
      ok = false;
      break;
    }
    L[j][j] = std::sqrt(s);
    for (int i = j + 1; i < 6; ++i) {
      double t = M[i][j];
      for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
      L[i][j] = t / L[j][j];
    }
  }
  if (ok) {
    double yv[6];
    for (int i = 0; i < 6; ++i) {
      double t = g[i];
      for (int k = 0; k < i; ++k) t -= L[i][k] * yv[k];
      yv[i] = t / L[i][i];
    }
    for (int i = 5; i >= 0; --i) {
      double t = yv[i];
      for (int k = i + 1; k < 6; ++k) t -= L[k][i] * x[k];
      x[i] = t / L[i][i];
    }
    return;
  }
  double A[6][7];
  for (int i = 0; i < 6; ++i) {
    for (int j = 0; j < 6; ++j) A[i][j] = M[i][j];
    A[i][6] = g[i];
  }
  for (int c = 0; c < 6; ++c) {
    int piv = c;
    for (int i = c + 1; i < 6; ++i)
      if (std::fabs(A[i][c]) > std::fabs(A[piv][c])) piv = i;
    if (piv != c)
      for (int j = 0; j < 7; ++j) std::swap(A[c][j], A[piv][j]);
    for (int i = c + 1; i < 6; ++i) {
      const double f = A[c][c] != 0 ? A[i][c] / A[c][c] : 0;
      for (int j = c; j < 7; ++j) A[i][j] -= f * A[c][j];
    }
  }
  for (int i = 5; i >= 0; --i) {
    double t = A[i][6];
    for (int k = i + 1; k < 6; ++k) t -= A[i][k] * x[k];
    x[i] = t / A[i][i];
  }
}

float restrict_angle(float a) {  // restrictTransform.m:24-25 in single precision
  const float tp = (float)(2 * M_PI);
  while (a > (float)M_PI) a = a - tp;
  while (a < -(float)M_PI) a = a + tp;
  return a;
}

}  // namespace

int dis_lm_step(disorder_ctx_s* ctx, const disorder_plan_s* plan, const LMSpec& s, float* T, float* w, uint8_t* cT,
                double* En_out, double* EnPrev_out) {
  const int S = plan->n_mot;
  const long long V = plan->V;
  const int N3 = plan->N[2];
  int n3_lo = s.n3_lo, n3_hi = s.n3_hi;
  if (n3_hi <= 0) {
    n3_lo = 0;
    n3_hi = N3;
  }
  if (n3_lo < 0 || n3_hi > N3 || n3_lo >= n3_hi) return dis_set_error(ctx, DISORDER_BAD_ARG, "LM: bad readout range");
  const int N3c = n3_hi - n3_lo;
  const double NElY = (double)plan->n_samples * N3 * s.C;  // numel(y) before the crop (LMsolver.m:32)
  const long long ny = plan->n_samples * (long long)N3 * s.C;
  int ha[21][2];
  ha_pairs(ha);
  std::vector<uint8_t> cTFull(cT, cT + S), flagw(S, 0);
  std::vector<int> act;
  for (int q = 0; q < S; ++q)
    if (!cTFull[q]) act.push_back(q);
  std::vector<double> EnPrev(S, 0.0), En(S, 0.0), dG((size_t)S * 6, 0.0), dH((size_t)S * 21, 0.0);
  std::vector<float> dGEff((size_t)S * 6, 0.f);
  // solver buffers: residual and the 6 encoded derivatives in the y layout
  const size_t need = sizeof(float2) * 7 * (size_t)ny + (1 << 20);
  Workspace sw;
  DIS_TRY(dis_workspace2(ctx, need, &sw));
  float2* rbuf = sw.take<float2>(ny);
  float2* gbuf = sw.take<float2>(6 * ny);
  if (!rbuf || !gbuf) return dis_set_error(ctx, DISORDER_OOM, "LM workspace");
  // per-slot operator memory: z, yB(2), w1, w2, G(6) + coil stage
  const size_t coil = (size_t)s.C * plan->N[0] * plan->N[1] * N3c * sizeof(float2);
  const size_t per_slot = 11 * (size_t)V * sizeof(float2) + coil + dis_table_bytes(plan, 1, true);
  const int ch = (int)std::max<size_t>(1, std::min<size_t>(std::max<size_t>(act.size(), 1), dis_budget_bytes() / per_slot));
  std::vector<double> sums;
  // ---- Jacobian (LMsolver.m:44-123)
  for (size_t c0 = 0; c0 < act.size(); c0 += ch) {
    const int n = (int)std::min<size_t>(ch, act.size() - c0);
    std::vector<int> st(act.begin() + c0, act.begin() + c0 + n);
    Workspace w0;
    DIS_TRY(dis_workspace(ctx, (size_t)n * per_slot + (1 << 20), &w0));
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w0, st, &d_seg));
    float2* z = w0.take<float2>((size_t)n * V);
    float2* yB = w0.take<float2>((size_t)2 * n * V);
    float2* w1 = w0.take<float2>((size_t)n * V);
    float2* w2 = w0.take<float2>((size_t)n * V);
    float2* G = w0.take<float2>((size_t)6 * n * V);
    float2* A = w0.take<float2>((size_t)n * s.C * plan->N[0] * plan->N[1] * N3c);
    if (!z || !yB || !w1 || !w2 || !G || !A) return dis_set_error(ctx, DISORDER_OOM, "LM workspace");
    std::vector<SlotParams> prm;
    dis_slot_params(T, S, st.data(), n, 1, &prm);
    Tables tb;
    DIS_TRY(dis_build_tables(ctx, plan, prm, true, &w0, &tb));
    DIS_TRY(dis_gradient(ctx, plan, s.x, 0, tb, z, yB, w1, w2, G));
    // r = encode(xT) - y (:72), the derivative encodes (:97-99)
    DIS_TRY(dis_encode_volumes(ctx, plan, z, d_seg, st, s.Sf, s.C, n3_lo, N3c, A, rbuf, plan->n_samples, n3_lo, N3,
                               s.y));
    for (int g = 0; g < 6; ++g)
      DIS_TRY(dis_encode_volumes(ctx, plan, G + (long long)g * n * V, d_seg, st, s.Sf, s.C, n3_lo, N3c, A,
                                 gbuf + (long long)g * ny, plan->n_samples, n3_lo, N3, nullptr));
    double* d_out = w0.take<double>((size_t)n * 28);
    if (!d_out) return dis_set_error(ctx, DISORDER_OOM, "LM workspace");
    DIS_TRY(dis_seg_sums(ctx, plan, d_seg, n, rbuf, gbuf, ny, plan->n_samples, n3_lo, N3c, N3, s.C, nullptr, d_out,
                         &w0));
    sums.assign((size_t)n * 28, 0.0);
    DIS_CUDA_TRY(cudaMemcpyAsync(sums.data(), d_out, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (double v : sums)
      if (!std::isfinite(v))
        return dis_set_error(ctx, DISORDER_NONFINITE, "LM: non-finite residual or Jacobian sums (non-finite y or x?)");
    for (int j = 0; j < n; ++j) {
      const int q = st[j];
      EnPrev[q] = sums[j * 28] / NElY;  // :82-83,93
      for (int g = 0; g < 6; ++g) dG[q * 6 + g] = sums[j * 28 + 1 + g];
      for (int h = 0; h < 21; ++h) dH[q * 21 + h] = sums[j * 28 + 7 + h];
    }
  }
  // ---- damping loop (:126-215)
  En = EnPrev;
  std::vector<float> Tcur(T, T + 6 * S), Tup(6 * S), Tupr(6 * S);
  int guard = 0;
  while (true) {
    for (int a = 0; a < S; ++a) {
      if (cTFull[a] || !(w[a] < 1e10f)) continue;
      double M[6][6], g[6], x6[6];
      for (int h = 0; h < 21; ++h) {
        const int p = ha[h][0], q = ha[h][1];
        const float v = (float)dH[a * 21 + h];  // dH is single in the reference
        if (p == q)
          M[p][q] = (double)((1.0f + w[a]) * v);
        else
          M[p][q] = M[q][p] = (double)v;
      }
      for (int k = 0; k < 6; ++k) g[k] = (double)(float)dG[a * 6 + k];
      solve6(M, g, x6);
      for (int k = 0; k < 6; ++k) dGEff[a * 6 + k] = -(s.winit / w[a]) * (float)x6[k];
    }
    for (int a = 0; a < S; ++a)
      for (int p = 0; p < 6; ++p) {
        Tupr[p * S + a] = dGEff[a * 6 + p];
        float v = Tcur[p * S + a] + Tupr[p * S + a];
        if (p >= 3) v = restrict_angle(v);
        Tup[p * S + a] = v;
      }
    std::vector<int> ev;
    for (int q = 0; q < S; ++q)
      if (!(cTFull[q] || flagw[q])) ev.push_back(q);
    // energies with the candidate motion (:147-194)
    const size_t per_e = (size_t)V * sizeof(float2) + coil + dis_table_bytes(plan, 1, false);
    const int che = (int)std::max<size_t>(1, std::min<size_t>(std::max<size_t>(ev.size(), 1), dis_budget_bytes() / per_e));
    for (size_t c0 = 0; c0 < ev.size(); c0 += che) {
      const int n = (int)std::min<size_t>(che, ev.size() - c0);
      std::vector<int> st(ev.begin() + c0, ev.begin() + c0 + n);
      Workspace w0;
      DIS_TRY(dis_workspace(ctx, (size_t)n * per_e + (1 << 20), &w0));
      int* d_seg = nullptr;
      DIS_TRY(dis_upload_ints(ctx, &w0, st, &d_seg));
      float2* z = w0.take<float2>((size_t)n * V);
      float2* A = w0.take<float2>((size_t)n * s.C * plan->N[0] * plan->N[1] * N3c);
      if (!z || !A) return dis_set_error(ctx, DISORDER_OOM, "LM workspace");
      std::vector<SlotParams> prm;
      dis_slot_params(Tup.data(), S, st.data(), n, 1, &prm);
      Tables tb;
      DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w0, &tb));
      DIS_TRY(dis_forward_transform(ctx, plan, s.x, 0, z, tb, 1, nullptr));
      DIS_TRY(dis_encode_volumes(ctx, plan, z, d_seg, st, s.Sf, s.C, n3_lo, N3c, A, rbuf, plan->n_samples, n3_lo, N3,
                                 s.y));
      double* d_out = w0.take<double>((size_t)n * 28);
      if (!d_out) return dis_set_error(ctx, DISORDER_OOM, "LM workspace");
      DIS_TRY(dis_seg_sums(ctx, plan, d_seg, n, rbuf, nullptr, 0, plan->n_samples, n3_lo, N3c, N3, s.C, nullptr,
                           d_out, &w0));
      sums.assign((size_t)n * 28, 0.0);
      DIS_CUDA_TRY(cudaMemcpyAsync(sums.data(), d_out, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      for (int j = 0; j < n; ++j) En[st[j]] = sums[j * 28] / NElY;
    }
    for (int q = 0; q < S; ++q)
      if (w[q] > 1e10f) En[q] = EnPrev[q];  // :195
    for (int q = 0; q < S; ++q)
      if (En[q] <= EnPrev[q]) flagw[q] = 1;  // :196
    bool all = true;
    for (int q = 0; q < S; ++q) all = all && flagw[q];
    if (!all) {  // :199-200
      for (int q = 0; q < S; ++q)
        if (En[q] > EnPrev[q] && !cTFull[q]) w[q] = w[q] * 2.0f;
    } else {  // :201-213
      for (int q = 0; q < S; ++q)
        if (!cTFull[q]) w[q] = w[q] / 1.2f;
      for (int q = 0; q < S; ++q)
        if (w[q] < 1e-8f) w[q] = 1.2f * w[q];
      Tcur = Tup;
      for (int q = 0; q < S; ++q) {
        float tm = 0.f, rm = 0.f;
        for (int p = 0; p < 3; ++p) tm = std::max(tm, std::fabs(Tupr[p * S + q]));
        for (int p = 3; p < 6; ++p) rm = std::max(rm, std::fabs(180.0f * Tupr[p * S + q] / (float)M_PI));
        if (tm < s.tL[0] && rm < s.tL[1]) cTFull[q] = 1;
      }
      break;
    }
    if (++guard > 200) return dis_set_error(ctx, DISORDER_TIMEOUT, "LM: damping loop did not settle");
  }
  std::copy(Tcur.begin(), Tcur.end(), T);
  for (int q = 0; q < S; ++q) cT[q] = cTFull[q];
  if (En_out) std::copy(En.begin(), En.end(), En_out);
  if (EnPrev_out) std::copy(EnPrev.begin(), EnPrev.end(), EnPrev_out);
  return DISORDER_OK;
}
