// Phase factors of the sinc rigid transform
// (Methods/precomputeFactorsSincRigidTransform.m:42-125, gr=1, sh=1).
// Per-state scalars (wrapped angles, tan/sin/cos) are formed on the host in
// double precision; the per-element factors exp(i*phase) are evaluated on the
// device in double precision and rounded to single. The 1/N of the inverse
// DFT of the pass that applies a factor is folded into that factor.
#include <algorithm>
#include <cmath>

#include "fastpass.h"
#include "internal.h"

namespace {

const int TR0[3] = {0, 2, 1};  // tr(1,:) of sincRigidTransform.m:33 (0-based)
const int TR1[3] = {1, 0, 2};  // tr(2,:)

double wrap_to_pi(double x) {  // Mapping Toolbox wrapToPi, from its definition
  if (x < -M_PI || x > M_PI) {
    const double y = x + M_PI;
    double w = y - std::floor(y / (2 * M_PI)) * (2 * M_PI);
    if (w == 0 && y > 0) w = 2 * M_PI;
    return w - M_PI;
  }
  return x;
}

double wrap_to_pi_half(double x) {  // Methods/wrapToPiHalf.m:9-12
  double m = x - std::floor(x / M_PI) * M_PI;
  if (m > M_PI / 2) m -= M_PI;
  return m;
}

// e2/e3 tables: [slot][r][k], phase = coef[slot] * fl(rG[r] * kG[k]); k along the pass axis.
__global__ void shear_table_kernel(float2* __restrict__ tab, float2* __restrict__ gtab, int nk, int nr,
                                   const float* __restrict__ kG, const float* __restrict__ rG,
                                   const double* __restrict__ coef, const double* __restrict__ gcoef,
                                   int gsign, double invn, int n_slots) {
  const long long per = (long long)nk * nr;
  const long long tot = per * n_slots;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
    const int slot = (int)(e / per);
    const long long rem = e - slot * per;
    const int r = (int)(rem / nk), k = (int)(rem - (long long)r * nk);
    const float rk = __fmul_rn(rG[r], kG[k]);  // rkGrid is a single-precision product
    double s, c;
    sincos(coef[slot] * (double)rk, &s, &c);
    const float2 v = make_float2((float)(c * invn), (float)(s * invn));
    tab[e] = v;
    if (gtab) {
      // etg2 = i*g*rk*e2 (gsign=+1), etg3 = -i*g*rk*e3 (gsign=-1)
      const double a = gsign * gcoef[slot] * (double)rk;
      gtab[e] = make_float2((float)(-a * s * invn), (float)(a * c * invn));
    }
  }
}

__global__ void trans_table_kernel(float2* __restrict__ tab, int nk, const float* __restrict__ kG,
                                   const double* __restrict__ t, int n_slots) {
  const long long tot = (long long)nk * n_slots;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
    const int slot = (int)(e / nk), k = (int)(e - (long long)slot * nk);
    double s, c;
    sincos(t[slot] * (double)kG[k], &s, &c);
    tab[e] = make_float2((float)c, (float)s);
  }
}

// Seeds of the coefficient invn * exp(i*phi*kG[k]) along a pass axis of
// even length N = F1*F2 whose kGrid is linear, kG[k] = alpha*kv(k) with
// kv(k) = k for k < N/2 and k - N beyond, for phi = coef[slot]*rG[row] +
// t[slot] (either term may be absent). Row `row` of slot `slot` holds
//   [j]        invn * exp(i*phi*alpha*j)                   j < F1
//   [F1 + j]   invn * exp(i*phi*alpha*(j + F1*k2h - N))    j < F1, k2h = ceil(F2/2)
//   [2*F1]     exp(i*phi*alpha*F1)                         (the step in k2)
//   [2*F1+1]   0                                           (pads rows to 16 bytes)
// so that the coefficient of frequency k = j + F1*k2 is lo[j]*step^k2 on the
// non-negative side and hi[j]*step^(k2-k2h) on the negative side. The phase
// is formed in double precision from rG*alpha*kv, where the e2/e3 tables
// round the product rG*kG to single first (Methods/generateTransformGrids.m:57-62).
__global__ void seed_table_kernel(float2* __restrict__ tab, int nr, int sw, int F1, int N, int k2h, double alpha,
                                  double invn, const float* __restrict__ rG, const double* __restrict__ coef,
                                  const double* __restrict__ t, int n_slots) {
  const long long per = (long long)nr * sw;
  const long long tot = per * n_slots;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
    const int slot = (int)(e / per);
    const long long rem = e - slot * per;
    const int r = (int)(rem / sw), j = (int)(rem - (long long)r * sw);
    double phi = 0.0;
    if (coef) phi += coef[slot] * (double)rG[r];
    if (t) phi += t[slot];
    double kv, sc = invn;
    if (j < F1) {
      kv = j;
    } else if (j < 2 * F1) {
      kv = (double)(j - F1) + (double)F1 * k2h - N;
    } else if (j == 2 * F1) {
      kv = F1;
      sc = 1.0;
    } else {
      tab[e] = make_float2(0.f, 0.f);
      continue;
    }
    double s, c;
    sincos(phi * alpha * kv, &s, &c);
    tab[e] = make_float2((float)(c * sc), (float)(s * sc));
  }
}

// Seed tables of the pipelined passes (left null, and the passes on the
// e1/e2/e3 tables, unless every axis has a pipelined kernel and a linear
// kGrid). d: the per-slot scalars [what][m][slot] of dis_build_tables.
int build_seeds(disorder_ctx_s* ctx, const disorder_plan_s* plan, const double* d, int ns, Workspace* ws,
                Tables* tb) {
  if (!dis_use_fast() || !dis_use_pipe()) return DISORDER_OK;
  const int* N = plan->N;
  int F1[3], F2[3];
  for (int a = 0; a < 3; ++a)
    if (!dis_fast_factor(N[a], &F1[a], &F2[a]) || !plan->k_linear[a]) return DISORDER_OK;
  for (int a = 0; a < 3; ++a) tb->sdw[a] = 2 * F1[a] + 2;
  const int blocks = 2 * ctx->sm_count;
  auto make = [&](int ax, int nr, const float* rG, const double* coef, const double* t, long long* stride) -> float2* {
    *stride = (long long)nr * tb->sdw[ax];
    float2* p = ws->take<float2>((size_t)(*stride) * ns);
    if (!p) return nullptr;
    seed_table_kernel<<<blocks, 256, 0, ctx->stream>>>(p, nr, tb->sdw[ax], F1[ax], N[ax], (F2[ax] + 1) / 2,
                                                       plan->k_alpha[ax], 1.0 / N[ax], rG, coef, t, ns);
    dis_count(ctx);
    return p;
  };
  for (int m = 0; m < 3; ++m) {
    const int a1 = TR0[m], a2 = TR1[m];
    tb->sd2[m] = make(a1, N[a2], plan->d_rG[a2], d + (0 * 3 + m) * ns, nullptr, &tb->sd2s[m]);
    tb->sd3[m] = make(a2, N[a1], plan->d_rG[a1], d + (1 * 3 + m) * ns, nullptr, &tb->sd3s[m]);
    if (!tb->sd2[m] || !tb->sd3[m]) return dis_set_error(ctx, DISORDER_OOM, "tables: workspace too small");
  }
  tb->sd2t = make(TR0[2], N[TR1[2]], plan->d_rG[TR1[2]], d + (0 * 3 + 2) * ns, d + (4 * 3 + 1) * ns, &tb->sd2ts);
  if (!tb->sd2t) return dis_set_error(ctx, DISORDER_OOM, "tables: workspace too small");
  for (int a = 0; a < 3; ++a) {
    tb->sd1[a] = make(a, 1, nullptr, nullptr, d + (4 * 3 + a) * ns, &tb->sd1s[a]);
    if (!tb->sd1[a]) return dis_set_error(ctx, DISORDER_OOM, "tables: workspace too small");
  }
  return DISORDER_OK;
}

}  // namespace

// Per-state scalars of one transform (precomputeFactorsSincRigidTransform.m:45-65)
// from T(s, :) of an n_states x 6 parameter-major array.
static void slot_params_one(const float* T, int n_states, int s, int di, SlotParams* p) {
  const double sd = (di == 1) ? -1.0 : 1.0;    // (-1)^di
  const double sdm = (di == 1) ? 1.0 : -1.0;   // (-1)^(di-1)
  for (int a = 0; a < 3; ++a) p->t[a] = sd * (double)T[a * n_states + s];
  for (int m = 0; m < 3; ++m) {
    double th = wrap_to_pi((double)T[(3 + m) * n_states + s]);
    p->flip[m] = std::fabs(th) > M_PI / 2 ? 1 : 0;
    th = wrap_to_pi_half(th);
    const double t2 = std::tan(th / 2);
    p->tau[m] = sdm * t2;
    p->sig[m] = sd * std::sin(th);
    p->g2[m] = (1 + t2 * t2) / 2;
    p->g3[m] = std::cos(th);
  }
}

void dis_slot_params_into(const float* T, int n_states, int di, SlotParams* out) {
  for (int s = 0; s < n_states; ++s) slot_params_one(T, n_states, s, di, &out[s]);
}

void dis_slot_params(const float* T, int n_states, const int* slots, int n_slots, int di,
                     std::vector<SlotParams>* out) {
  out->resize(n_slots);
  for (int j = 0; j < n_slots; ++j) slot_params_one(T, n_states, slots ? slots[j] : j, di, &(*out)[j]);
}

// Places the forward/inverse tables of ns slots (no derivative factors, no
// seeds) in ws: the per-slot scalars d, then e2/e3 per rotation, then e1 per
// axis. The one layout both dis_static_table_bytes and dis_build_tables_into
// use. Returns false when ws runs out.
static bool static_table_layout(const disorder_plan_s* plan, int ns, Workspace* ws, Tables* tb, double** d) {
  const int* N = plan->N;
  *d = ws->take<double>(15 * (size_t)ns);
  if (!*d) return false;
  for (int m = 0; m < 3; ++m) {
    const int a1 = TR0[m], a2 = TR1[m];
    tb->e2s[m] = (long long)N[a1] * N[a2];
    tb->e3s[m] = (long long)N[a2] * N[a1];
    tb->e2[m] = ws->take<float2>(tb->e2s[m] * ns);
    tb->e3[m] = ws->take<float2>(tb->e3s[m] * ns);
    tb->g2[m] = tb->g3[m] = nullptr;
    if (!tb->e2[m] || !tb->e3[m]) return false;
  }
  for (int a = 0; a < 3; ++a) {
    tb->e1s[a] = N[a];
    tb->e1[a] = ws->take<float2>((size_t)N[a] * ns);
    if (!tb->e1[a]) return false;
  }
  return true;
}

size_t dis_static_table_bytes(const disorder_plan_s* plan, int ns) {
  // a counting workspace: a non-null base that is never dereferenced
  Workspace ws;
  ws.base = reinterpret_cast<char*>(256);
  ws.cap = ~size_t(0) >> 1;
  ws.off = 0;
  Tables tb;
  double* d = nullptr;
  static_table_layout(plan, ns, &ws, &tb, &d);
  return ws.off;
}

// Forward/inverse transform tables for ns <= kMaxStaticSlots slots placed in
// the caller's region [base, base+cap) with no heap use on the host or the
// device: the per-slot scalars are staged in a thread-local static array.
// Returns OOM when the tables do not fit in cap bytes. Flip-slot lists are not
// built (the caller rejects rotations beyond 90 degrees).
int dis_build_tables_into(disorder_ctx_s* ctx, const disorder_plan_s* plan, const SlotParams* sp, int ns,
                          char* base, size_t cap, Tables* tb) {
  if (ns < 1 || ns > kMaxStaticSlots) return dis_set_error(ctx, DISORDER_BAD_ARG, "tables: %d slots", ns);
  Workspace ws;
  ws.base = base;
  ws.cap = cap;
  ws.off = 0;
  const int* N = plan->N;
  double* d = nullptr;
  if (!static_table_layout(plan, ns, &ws, tb, &d)) return DISORDER_OOM;
  static thread_local double h[15 * kMaxStaticSlots];
  for (int j = 0; j < ns; ++j)
    for (int m = 0; m < 3; ++m) {
      h[(0 * 3 + m) * ns + j] = sp[j].tau[m];
      h[(1 * 3 + m) * ns + j] = sp[j].sig[m];
      h[(2 * 3 + m) * ns + j] = sp[j].g2[m];
      h[(3 * 3 + m) * ns + j] = sp[j].g3[m];
      h[(4 * 3 + m) * ns + j] = sp[j].t[m];
    }
  // a pageable-source copy is staged before the call returns
  DIS_CUDA_TRY(cudaMemcpyAsync(d, h, 15 * (size_t)ns * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  tb->n_slots = ns;
  const int blocks = 2 * ctx->sm_count;
  for (int m = 0; m < 3; ++m) {
    const int a1 = TR0[m], a2 = TR1[m];
    shear_table_kernel<<<blocks, 256, 0, ctx->stream>>>(tb->e2[m], nullptr, N[a1], N[a2], plan->d_kG[a1],
                                                        plan->d_rG[a2], d + (0 * 3 + m) * ns, d + (2 * 3 + m) * ns,
                                                        +1, 1.0 / N[a1], ns);
    shear_table_kernel<<<blocks, 256, 0, ctx->stream>>>(tb->e3[m], nullptr, N[a2], N[a1], plan->d_kG[a2],
                                                        plan->d_rG[a1], d + (1 * 3 + m) * ns, d + (3 * 3 + m) * ns,
                                                        -1, 1.0 / N[a2], ns);
    dis_count(ctx, 2);
  }
  for (int a = 0; a < 3; ++a) {
    trans_table_kernel<<<blocks, 256, 0, ctx->stream>>>(tb->e1[a], N[a], plan->d_kG[a], d + (4 * 3 + a) * ns, ns);
    dis_count(ctx);
  }
  for (int m = 0; m < 3; ++m) {
    tb->any_flip[m] = false;
    tb->d_flip_slots[m] = nullptr;
  }
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int dis_build_tables(disorder_ctx_s* ctx, const disorder_plan_s* plan, const std::vector<SlotParams>& sp,
                     bool with_grad, Workspace* ws, Tables* tb) {
  const int ns = (int)sp.size();
  tb->n_slots = ns;
  if (ns == 0) return DISORDER_OK;
  const int* N = plan->N;
  // per-slot scalars: [what][m][slot]
  std::vector<double> h(ns * 15);
  for (int j = 0; j < ns; ++j)
    for (int m = 0; m < 3; ++m) {
      h[(0 * 3 + m) * ns + j] = sp[j].tau[m];
      h[(1 * 3 + m) * ns + j] = sp[j].sig[m];
      h[(2 * 3 + m) * ns + j] = sp[j].g2[m];
      h[(3 * 3 + m) * ns + j] = sp[j].g3[m];
      h[(4 * 3 + m) * ns + j] = sp[j].t[m];
    }
  double* d = ws->take<double>(h.size());
  if (!d) return dis_set_error(ctx, DISORDER_OOM, "tables: workspace too small");
  DIS_CUDA_TRY(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  const int blocks = 2 * ctx->sm_count;
  for (int m = 0; m < 3; ++m) {
    const int a1 = TR0[m], a2 = TR1[m];
    tb->e2s[m] = (long long)N[a1] * N[a2];
    tb->e3s[m] = (long long)N[a2] * N[a1];
    tb->e2[m] = ws->take<float2>(tb->e2s[m] * ns);
    tb->e3[m] = ws->take<float2>(tb->e3s[m] * ns);
    if (with_grad) {
      tb->g2[m] = ws->take<float2>(tb->e2s[m] * ns);
      tb->g3[m] = ws->take<float2>(tb->e3s[m] * ns);
    } else {
      tb->g2[m] = tb->g3[m] = nullptr;
    }
    if (!tb->e2[m] || !tb->e3[m] || (with_grad && (!tb->g2[m] || !tb->g3[m])))
      return dis_set_error(ctx, DISORDER_OOM, "tables: workspace too small");
    // e2{m}: k along a1, r along a2
    shear_table_kernel<<<blocks, 256, 0, ctx->stream>>>(tb->e2[m], tb->g2[m], N[a1], N[a2], plan->d_kG[a1],
                                                        plan->d_rG[a2], d + (0 * 3 + m) * ns, d + (2 * 3 + m) * ns,
                                                        +1, 1.0 / N[a1], ns);
    // e3{m}: k along a2, r along a1
    shear_table_kernel<<<blocks, 256, 0, ctx->stream>>>(tb->e3[m], tb->g3[m], N[a2], N[a1], plan->d_kG[a2],
                                                        plan->d_rG[a1], d + (1 * 3 + m) * ns, d + (3 * 3 + m) * ns,
                                                        -1, 1.0 / N[a2], ns);
    dis_count(ctx, 2);
  }
  for (int a = 0; a < 3; ++a) {
    tb->e1s[a] = N[a];
    tb->e1[a] = ws->take<float2>((size_t)N[a] * ns);
    if (!tb->e1[a]) return dis_set_error(ctx, DISORDER_OOM, "tables: workspace too small");
    trans_table_kernel<<<blocks, 256, 0, ctx->stream>>>(tb->e1[a], N[a], plan->d_kG[a], d + (4 * 3 + a) * ns, ns);
    dis_count(ctx);
  }
  DIS_TRY(build_seeds(ctx, plan, d, ns, ws, tb));
  for (int m = 0; m < 3; ++m) {
    tb->flip_slots[m].clear();
    for (int j = 0; j < ns; ++j)
      if (sp[j].flip[m]) tb->flip_slots[m].push_back(j);
    tb->any_flip[m] = !tb->flip_slots[m].empty();
    tb->d_flip_slots[m] = nullptr;
    if (tb->any_flip[m]) {
      tb->d_flip_slots[m] = ws->take<int>(tb->flip_slots[m].size());
      if (!tb->d_flip_slots[m]) return dis_set_error(ctx, DISORDER_OOM, "tables: workspace too small");
      DIS_CUDA_TRY(cudaMemcpyAsync(tb->d_flip_slots[m], tb->flip_slots[m].data(),
                                   tb->flip_slots[m].size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    }
  }
  // (pageable-source async copies are staged before they return, so the
  // host vectors above may go out of scope)
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

// ---------------------------------------------------------------- factors as arrays
namespace {

// out[(i + Nlo*j) + Nlo*Nhi*s] = exp(i * coef[s] * rk), rk the single-precision
// product rG[ra][.] * kG[ka][.] over the two dims lo < hi of {ra, ka}
__global__ void shear_factor_kernel(const float* __restrict__ rG, const float* __restrict__ kG, int Nlo, int Nhi,
                                    int r_is_lo, const double* __restrict__ coef, int S, float2* __restrict__ out) {
  const long long n = (long long)Nlo * Nhi * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % Nlo);
    const long long q = e / Nlo;
    const int j = (int)(q % Nhi);
    const int s = (int)(q / Nhi);
    const float rk = r_is_lo ? rG[i] * kG[j] : rG[j] * kG[i];
    double sn, cs;
    sincos(coef[s] * (double)rk, &sn, &cs);
    out[e] = make_float2((float)cs, (float)sn);
  }
}

// out[k + N*s] = exp(i * t[s] * kG[k])
__global__ void ramp_factor_kernel(const float* __restrict__ kG, int N, const double* __restrict__ t, int S,
                                   float2* __restrict__ out) {
  const long long n = (long long)N * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e % N);
    const int s = (int)(e / N);
    double sn, cs;
    sincos(t[s] * (double)kG[k], &sn, &cs);
    out[e] = make_float2((float)cs, (float)sn);
  }
}

}  // namespace

extern "C" int disorder_precompute_factors(disorder_ctx ctx, disorder_plan plan, const float* T, int32_t n_states,
                                           int32_t di, void* e1, void* e2, void* e3, uint8_t* flip) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!plan || plan->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan");
  if (!T || n_states < 1 || (di != 0 && di != 1))
    return dis_set_error(ctx, DISORDER_BAD_ARG, "precompute factors: bad arguments");
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  const int S = n_states;
  std::vector<SlotParams> prm;
  dis_slot_params(T, S, nullptr, S, di, &prm);
  if (flip)
    for (int m = 0; m < 3; ++m)
      for (int s = 0; s < S; ++s) flip[m * S + s] = (uint8_t)prm[s].flip[m];
  // per-state coefficients: t (e1), tau (e2), sig (e3) for the 3 blocks
  std::vector<double> h((size_t)9 * S);
  for (int m = 0; m < 3; ++m)
    for (int s = 0; s < S; ++s) {
      h[(size_t)(0 * 3 + m) * S + s] = prm[s].t[m];
      h[(size_t)(1 * 3 + m) * S + s] = prm[s].tau[m];
      h[(size_t)(2 * 3 + m) * S + s] = prm[s].sig[m];
    }
  Workspace ws;
  DIS_TRY(dis_small(ctx, &ws));
  double* d = ws.take<double>(h.size());
  if (!d) return dis_set_error(ctx, DISORDER_OOM, "precompute factors: scratch");
  DIS_CUDA_TRY(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  const int* N = plan->N;
  // rkGrid{1}{m}: rG along per(2,m), kG along per(1,m); rkGrid{2}{m} the
  // reverse (Methods/generateTransformGrids.m:57-62, per = [1 3 2; 2 1 3])
  const int per[2][3] = {{0, 2, 1}, {1, 0, 2}};
  long long off2 = 0;
  long long off1 = 0;
  for (int m = 0; m < 3; ++m) {
    if (e1) {
      ramp_factor_kernel<<<256, 256, 0, ctx->stream>>>(plan->d_kG[m], N[m], d + (size_t)m * S, S,
                                                       (float2*)e1 + off1);
      dis_count(ctx);
    }
    off1 += (long long)N[m] * S;
    for (int which = 0; which < 2; ++which) {
      void* out = which == 0 ? e2 : e3;
      if (!out) continue;
      const int ra = which == 0 ? per[1][m] : per[0][m];
      const int ka = which == 0 ? per[0][m] : per[1][m];
      const int lo = std::min(ra, ka), hi = std::max(ra, ka);
      shear_factor_kernel<<<256, 256, 0, ctx->stream>>>(plan->d_rG[ra], plan->d_kG[ka], N[lo], N[hi], ra == lo ? 1 : 0,
                                                        d + (size_t)((1 + which) * 3 + m) * S, S,
                                                        (float2*)out + off2);
      dis_count(ctx);
    }
    const int a = m == 2 ? 1 : 0, b = m == 0 ? 1 : 2;  // blocks span dims {0,1}, {0,2}, {1,2}
    off2 += (long long)N[a] * N[b] * S;
  }
  DIS_CUDA_TRY(cudaGetLastError());
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}
