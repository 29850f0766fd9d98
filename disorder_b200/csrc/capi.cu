// C ABI of libdisorder: contexts, workspaces, plans and the entry points
// declared in include/disorder.h.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "encoding.h"
#include "internal.h"
#include "solvers.h"

int dis_set_error(disorder_ctx_s* ctx, int status, const char* fmt, ...) {
  if (ctx) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
    va_end(ap);
  }
  return status;
}

static int grow(disorder_ctx_s* ctx, void** buf, size_t* cap, size_t bytes) {
  if (bytes <= *cap && *buf) return DISORDER_OK;
  if (ctx->fault == DISORDER_FAULT_OOM) {
    ctx->fault = DISORDER_FAULT_NONE;
    return dis_set_error(ctx, DISORDER_OOM, "cudaMalloc of %zu bytes failed: injected fault", bytes);
  }
  if (*buf) {
    DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    cudaFree(*buf);
    *buf = nullptr;
    *cap = 0;
  }
  const size_t want = std::max<size_t>(bytes + bytes / 8, 1 << 20);
  cudaError_t e = cudaMalloc(buf, want);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *buf = nullptr;
    return dis_set_error(ctx, DISORDER_OOM, "cudaMalloc of %zu bytes failed: %s", want, cudaGetErrorString(e));
  }
  *cap = want;
  return DISORDER_OK;
}

int dis_workspace(disorder_ctx_s* ctx, size_t bytes, Workspace* ws) {
  DIS_TRY(grow(ctx, &ctx->ws, &ctx->ws_bytes, bytes));
  ws->base = (char*)ctx->ws;
  ws->cap = ctx->ws_bytes;
  ws->off = 0;
  return DISORDER_OK;
}

int dis_workspace2(disorder_ctx_s* ctx, size_t bytes, Workspace* ws) {
  DIS_TRY(grow(ctx, &ctx->ws2, &ctx->ws2_bytes, bytes));
  ws->base = (char*)ctx->ws2;
  ws->cap = ctx->ws2_bytes;
  ws->off = 0;
  return DISORDER_OK;
}

int dis_small(disorder_ctx_s* ctx, Workspace* ws) {
  DIS_TRY(grow(ctx, &ctx->small, &ctx->small_bytes, 16u << 20));
  ws->base = (char*)ctx->small;
  ws->cap = ctx->small_bytes;
  ws->off = 0;
  return DISORDER_OK;
}

int dis_ctas_per_sm(const void* fn, int threads, size_t dyn_smem) {
  cudaFuncAttributes fa;
  int dev = 0, smem_sm = 0, res_blk = 0, regs_sm = 0, thr_sm = 0, blk_sm = 0;
  if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&res_blk, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&blk_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev) != cudaSuccess || threads <= 0) {
    cudaGetLastError();
    return 0;
  }
  const long long smem_blk = (long long)dyn_smem + (long long)fa.sharedSizeBytes + res_blk;
  const int warps = (threads + 31) / 32;
  const long long regs_blk = (long long)warps * 32 * ((fa.numRegs + 7) / 8 * 8);  // 8-register granules
  long long n = std::min<long long>(thr_sm / threads, blk_sm);
  if (smem_blk > 0) n = std::min<long long>(n, smem_sm / smem_blk);
  if (regs_blk > 0) n = std::min<long long>(n, regs_sm / regs_blk);
  return (int)std::max<long long>(n, 0);
}

static bool use_pool() {
  static const bool v = [] {
    const char* e = std::getenv("DISORDER_POOL");
    return !(e && e[0] == '0');
  }();
  return v;
}

#define CTX_CHECK(ctx) \
  if (!(ctx)) return DISORDER_BAD_ARG
#define DEV_GUARD(ctx) DIS_CUDA_TRY(cudaSetDevice((ctx)->device))

extern "C" {

int disorder_ctx_create(int device, disorder_ctx* out) {
  if (!out) return DISORDER_BAD_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    cudaGetLastError();
    return DISORDER_CUDA_ERR;
  }
  disorder_ctx_s* ctx = new disorder_ctx_s();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ctx;
    return DISORDER_CUDA_ERR;
  }
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  ctx->smem_optin = optin;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return DISORDER_CUDA_ERR;
  }
  ctx->own_stream = true;
  // keep memory freed to the device's default pool (disorder_free) cached
  // for reuse instead of returning it to the driver at each synchronisation
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    // DISORDER_POOL_RESERVE_GB: grow the pool once, now, by allocating and
    // freeing that much, so that later allocations of varying sizes are
    // carved from memory it holds instead of mapping more in mid-run
    const char* e = std::getenv("DISORDER_POOL_RESERVE_GB");
    const double gb = e ? std::atof(e) : 0.0;
    if (use_pool() && gb > 0) {
      void* p = nullptr;
      if (cudaMallocAsync(&p, (size_t)(gb * (1ull << 30)), ctx->stream) == cudaSuccess) {
        cudaFreeAsync(p, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
      }
    }
  }
  cudaGetLastError();
  {  // DISORDER_SUM_COIL=1: new contexts start with the sample-sum coil stage
    const char* e = std::getenv("DISORDER_SUM_COIL");
    ctx->tune_coil = (e && e[0] == '1') ? 1 : 0;
  }
  // the static scratch of disorder_sinc_rigid_transform_static: resolving its
  // address here loads its module and commits it on this device, so that
  // entry point makes no allocation (a failure only disables that entry point)
  dis_static_scratch_resolve(&ctx->static_scratch, &ctx->static_scratch_bytes);
  if (cudaMalloc(&ctx->d_err, 256) != cudaSuccess || cudaMemset(ctx->d_err, 0, 256) != cudaSuccess) {
    cudaGetLastError();
    if (ctx->d_err) cudaFree(ctx->d_err);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return DISORDER_OOM;
  }
  *out = ctx;
  return DISORDER_OK;
}

int disorder_ctx_destroy(disorder_ctx ctx) {
  CTX_CHECK(ctx);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->ws) cudaFree(ctx->ws);
  if (ctx->ws2) cudaFree(ctx->ws2);
  if (ctx->small) cudaFree(ctx->small);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return DISORDER_OK;
}

const char* disorder_last_error(disorder_ctx ctx) { return ctx ? ctx->err : "null context"; }

int disorder_ctx_set_stream(disorder_ctx ctx, void* s) {
  CTX_CHECK(ctx);
  DEV_GUARD(ctx);
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  if (s) {
    ctx->stream = (cudaStream_t)s;
    ctx->own_stream = false;
  } else {
    DIS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    ctx->own_stream = true;
  }
  return DISORDER_OK;
}

void* disorder_ctx_get_stream(disorder_ctx ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int disorder_synchronize(disorder_ctx ctx) {
  CTX_CHECK(ctx);
  DEV_GUARD(ctx);
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  // err[0]: a bounded in-kernel wait that ran out (the kernel stopped early);
  // err[1]: the site of a device index check that failed (the access skipped)
  int err[2] = {0, 0};
  DIS_CUDA_TRY(cudaMemcpy(err, ctx->d_err, sizeof(err), cudaMemcpyDeviceToHost));
  if (err[0] || err[1]) DIS_CUDA_TRY(cudaMemset(ctx->d_err, 0, sizeof(err)));
  if (err[0])
    return dis_set_error(ctx, DISORDER_TIMEOUT, "a TMA tile wait in a line pass ran out; results are incomplete");
  if (err[1])
    return dis_set_error(ctx, DISORDER_BAD_ARG, "a device index check failed (site %d): an index outside its "
                         "array was skipped; results are incomplete", err[1]);
  return DISORDER_OK;
}

int disorder_malloc(disorder_ctx ctx, size_t bytes, void** dptr) {
  CTX_CHECK(ctx);
  if (!dptr) return dis_set_error(ctx, DISORDER_BAD_ARG, "malloc: null output");
  DEV_GUARD(ctx);
  // stream-ordered: no device-wide synchronisation, pooled reuse
  // (DISORDER_POOL=0: plain cudaMalloc / cudaFree)
  cudaError_t e = use_pool() ? cudaMallocAsync(dptr, std::max<size_t>(bytes, 1), ctx->stream)
                             : cudaMalloc(dptr, std::max<size_t>(bytes, 1));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return dis_set_error(ctx, DISORDER_OOM, "cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e));
  }
  return DISORDER_OK;
}

int disorder_free(disorder_ctx ctx, void* dptr) {
  CTX_CHECK(ctx);
  DEV_GUARD(ctx);
  if (!dptr) return DISORDER_OK;
  if (use_pool()) {
    DIS_CUDA_TRY(cudaFreeAsync(dptr, ctx->stream));
  } else {
    DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    DIS_CUDA_TRY(cudaFree(dptr));
  }
  return DISORDER_OK;
}

int disorder_memcpy_h2d(disorder_ctx ctx, void* dst, const void* src, size_t bytes) {
  CTX_CHECK(ctx);
  DEV_GUARD(ctx);
  DIS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

int disorder_memcpy_d2h(disorder_ctx ctx, void* dst, const void* src, size_t bytes) {
  CTX_CHECK(ctx);
  DEV_GUARD(ctx);
  DIS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  DIS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return DISORDER_OK;
}

int disorder_upload(disorder_ctx ctx, const void* host, size_t bytes, void** dptr) {
  CTX_CHECK(ctx);
  if (!dptr || (!host && bytes)) return dis_set_error(ctx, DISORDER_BAD_ARG, "upload: null argument");
  *dptr = nullptr;
  void* d = nullptr;
  DIS_TRY(disorder_malloc(ctx, bytes, &d));
  const int st = bytes ? disorder_memcpy_h2d(ctx, d, host, bytes) : DISORDER_OK;
  if (st != DISORDER_OK) {
    disorder_free(ctx, d);
    return st;
  }
  *dptr = d;
  return DISORDER_OK;
}

int disorder_download(disorder_ctx ctx, const void* dptr, void* host, size_t bytes) {
  CTX_CHECK(ctx);
  if (!bytes) return DISORDER_OK;
  if (!dptr || !host) return dis_set_error(ctx, DISORDER_BAD_ARG, "download: null argument");
  return disorder_memcpy_d2h(ctx, host, dptr, bytes);
}

int disorder_memcpy_d2d(disorder_ctx ctx, void* dst, const void* src, size_t bytes) {
  CTX_CHECK(ctx);
  DEV_GUARD(ctx);
  DIS_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  return DISORDER_OK;
}

int disorder_memset(disorder_ctx ctx, void* dst, int value, size_t bytes) {
  CTX_CHECK(ctx);
  DEV_GUARD(ctx);
  DIS_CUDA_TRY(cudaMemsetAsync(dst, value, bytes, ctx->stream));
  return DISORDER_OK;
}

int64_t disorder_kernel_launches(disorder_ctx ctx) { return ctx ? ctx->launches : -1; }

int disorder_ctx_inject_fault(disorder_ctx ctx, int32_t fault) {
  CTX_CHECK(ctx);
  if (fault < DISORDER_FAULT_NONE || fault > DISORDER_FAULT_OOM)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "inject_fault: unknown fault %d", fault);
  ctx->fault = fault;
  return DISORDER_OK;
}

int disorder_ctx_set_precision(disorder_ctx ctx, int32_t mode) {
  CTX_CHECK(ctx);
  if (mode < DISORDER_PRECISION_FP32 || mode > DISORDER_PRECISION_TF32X3)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "set_precision: unknown mode %d", mode);
  ctx->precision = mode;
  return DISORDER_OK;
}

int disorder_ctx_set_tuning(disorder_ctx ctx, int32_t key, int32_t value) {
  CTX_CHECK(ctx);
  switch (key) {
    case DISORDER_TUNE_TMA:
      if (value != 0 && value != 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "set_tuning: TMA is 0 or 1");
      ctx->tune_tma = value;
      return DISORDER_OK;
    case DISORDER_TUNE_COIL_STAGE:
      if (value != 0 && value != 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "set_tuning: coil stage is 0 or 1");
      ctx->tune_coil = value;
      return DISORDER_OK;
    default:
      return dis_set_error(ctx, DISORDER_BAD_ARG, "set_tuning: unknown key %d", key);
  }
}

int64_t disorder_workspace_bytes(disorder_ctx ctx) {
  return ctx ? (int64_t)(ctx->ws_bytes + ctx->ws2_bytes + ctx->small_bytes) : -1;
}

int disorder_event_record(disorder_ctx ctx, int32_t slot) {
  CTX_CHECK(ctx);
  if (slot < 0 || slot >= 16) return dis_set_error(ctx, DISORDER_BAD_ARG, "event slot %d", slot);
  DEV_GUARD(ctx);
  if (!ctx->ev[slot]) DIS_CUDA_TRY(cudaEventCreate(&ctx->ev[slot]));
  DIS_CUDA_TRY(cudaEventRecord(ctx->ev[slot], ctx->stream));
  return DISORDER_OK;
}

int disorder_event_elapsed(disorder_ctx ctx, int32_t a, int32_t b, float* ms) {
  CTX_CHECK(ctx);
  if (a < 0 || a >= 16 || b < 0 || b >= 16 || !ctx->ev[a] || !ctx->ev[b] || !ms)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "event_elapsed: bad slots");
  DEV_GUARD(ctx);
  DIS_CUDA_TRY(cudaEventSynchronize(ctx->ev[b]));
  DIS_CUDA_TRY(cudaEventElapsedTime(ms, ctx->ev[a], ctx->ev[b]));
  return DISORDER_OK;
}

// ---------------------------------------------------------------- plans
int disorder_plan_create(disorder_ctx ctx, const disorder_grid_desc* g, const disorder_sampling_desc* smp,
                         disorder_plan* out) {
  CTX_CHECK(ctx);
  if (!g || !smp || !out) return dis_set_error(ctx, DISORDER_BAD_ARG, "plan: null argument");
  *out = nullptr;
  DEV_GUARD(ctx);
  cudaGetLastError();  // the checks below read each call's own status, not an earlier one
  disorder_plan_s* p = new disorder_plan_s();
  p->ctx = ctx;
  auto fail = [&](int st) {
    disorder_plan_destroy(p);
    return st;
  };
  for (int m = 0; m < 3; ++m) {
    p->N[m] = g->N[m];
    if (g->N[m] < 1 || g->N[m] > 1024) return fail(dis_set_error(ctx, DISORDER_BAD_ARG, "plan: N[%d]=%d out of range", m, g->N[m]));
    if (!dis_make_fft_plan(g->N[m], &p->fft[m]))
      return fail(dis_set_error(ctx, DISORDER_BAD_ARG,
                                "plan: N[%d]=%d has a prime factor other than 2,3,5,7,11,13", m, g->N[m]));
    if (!g->rG[m] || !g->kG[m]) return fail(dis_set_error(ctx, DISORDER_BAD_ARG, "plan: missing grid %d", m));
    p->rG[m].assign(g->rG[m], g->rG[m] + g->N[m]);
    p->kG[m].assign(g->kG[m], g->kG[m] + g->N[m]);
    p->cent[m] = g->cent[m];
    // kG linear in the signed frequency (DC first, as generateTransformGrids
    // with sh=1 builds it): kG[k] ~ alpha * (k < N/2 ? k : k - N). The
    // pipelined passes then generate their phase factors from per-row seeds.
    const int n = p->N[m];
    double sxy = 0, sxx = 0;
    for (int k = 0; k < n; ++k) {
      const double kv = (k < n / 2 + (n & 1)) ? k : k - n;
      sxy += kv * p->kG[m][k];
      sxx += kv * kv;
    }
    p->k_alpha[m] = sxx > 0 ? sxy / sxx : 0.0;
    p->k_linear[m] = (n % 2 == 0) && sxx > 0;
    for (int k = 0; k < n && p->k_linear[m]; ++k) {
      const double kv = (k < n / 2) ? k : k - n;
      const double want = p->k_alpha[m] * kv, got = p->kG[m][k];
      if (std::fabs(got - want) > 4.0 * 1.2e-7 * std::fabs(want) + 1e-30) p->k_linear[m] = false;
    }
  }
  p->V = (long long)p->N[0] * p->N[1] * p->N[2];
  for (int m = 0; m < 3; ++m) {
    if (cudaMalloc(&p->d_kG[m], sizeof(float) * p->N[m]) != cudaSuccess ||
        cudaMalloc(&p->d_rG[m], sizeof(float) * p->N[m]) != cudaSuccess)
      return fail(dis_set_error(ctx, DISORDER_OOM, "plan: grid allocation"));
    if (cudaMemcpy(p->d_kG[m], p->kG[m].data(), sizeof(float) * p->N[m], cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(p->d_rG[m], p->rG[m].data(), sizeof(float) * p->N[m], cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(dis_set_error(ctx, DISORDER_CUDA_ERR, "plan: grid upload: %s", cudaGetErrorString(cudaGetLastError())));
    // twiddles exp(-2 pi i j / N) in double precision, rounded to single
    std::vector<float2> tw(p->N[m]);
    for (int j = 0; j < p->N[m]; ++j) {
      const double ang = -2.0 * M_PI * (double)j / (double)p->N[m];
      tw[j] = make_float2((float)std::cos(ang), (float)std::sin(ang));
    }
    if (cudaMalloc(&p->d_tw[m], sizeof(float2) * p->N[m]) != cudaSuccess)
      return fail(dis_set_error(ctx, DISORDER_OOM, "plan: twiddle allocation"));
    if (cudaMemcpy(p->d_tw[m], tw.data(), sizeof(float2) * p->N[m], cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(dis_set_error(ctx, DISORDER_CUDA_ERR, "plan: twiddle upload: %s", cudaGetErrorString(cudaGetLastError())));
  }
  // sampling
  if (smp->n_seg < 0 || smp->n_mot < 0 || smp->n_mot > smp->n_seg || !smp->seg_offsets)
    return fail(dis_set_error(ctx, DISORDER_BAD_ARG, "plan: bad segment counts"));
  p->n_seg = smp->n_seg;
  p->n_mot = smp->n_mot;
  p->seg_off.assign(smp->seg_offsets, smp->seg_offsets + smp->n_seg + 1);
  if (p->seg_off[0] != 0) return fail(dis_set_error(ctx, DISORDER_BAD_ARG, "plan: seg_offsets[0] must be 0"));
  for (int s = 0; s < p->n_seg; ++s)
    if (p->seg_off[s + 1] < p->seg_off[s]) return fail(dis_set_error(ctx, DISORDER_BAD_ARG, "plan: seg_offsets decrease"));
  const long long ns = p->seg_off[p->n_seg];
  p->n_samples = ns;
  if (ns > 0x7fffffffLL) return fail(dis_set_error(ctx, DISORDER_BAD_ARG, "plan: too many samples"));
  const int N1 = p->N[0], N2 = p->N[1];
  std::vector<int> segof(ns), rowptr((size_t)p->n_seg * (N1 + 1), 0), perm(ns);
  for (int s = 0; s < p->n_seg; ++s) {
    int* rp = rowptr.data() + (size_t)s * (N1 + 1);
    for (long long i = p->seg_off[s]; i < p->seg_off[s + 1]; ++i) {
      const int ky = smp->ky[i], kz = smp->kz[i];
      if (ky < 0 || ky >= N1 || kz < 0 || kz >= N2)
        return fail(dis_set_error(ctx, DISORDER_BAD_ARG, "plan: sample %lld row (%d,%d) outside %dx%d", i, ky, kz, N1, N2));
      segof[i] = s;
      rp[ky + 1]++;
    }
    for (int k = 0; k < N1; ++k) rp[k + 1] += rp[k];
    std::vector<int> fill(rp, rp + N1);
    for (long long i = p->seg_off[s]; i < p->seg_off[s + 1]; ++i) perm[p->seg_off[s] + fill[smp->ky[i]]++] = (int)i;
    for (int k = 0; k <= N1; ++k) rp[k] += (int)p->seg_off[s];
  }
  std::vector<int> kyq(ns), kzq(ns);
  for (long long q = 0; q < ns; ++q) {
    kyq[q] = smp->ky[perm[q]];
    kzq[q] = smp->kz[perm[q]];
  }
  auto up = [&](void** d, const void* h, size_t bytes) -> bool {
    if (cudaMalloc(d, std::max<size_t>(bytes, 4)) != cudaSuccess) return false;
    return !bytes || cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  if (!up((void**)&p->d_ky, smp->ky, sizeof(int) * ns) || !up((void**)&p->d_kz, smp->kz, sizeof(int) * ns) ||
      !up((void**)&p->d_seg_of, segof.data(), sizeof(int) * ns) ||
      !up((void**)&p->d_perm, perm.data(), sizeof(int) * ns) ||
      !up((void**)&p->d_kyq, kyq.data(), sizeof(int) * ns) || !up((void**)&p->d_kzq, kzq.data(), sizeof(int) * ns) ||
      !up((void**)&p->d_rowptr, rowptr.data(), sizeof(int) * rowptr.size()) ||
      !up((void**)&p->d_seg_off, p->seg_off.data(), sizeof(long long) * p->seg_off.size()))
    return fail(dis_set_error(ctx, DISORDER_OOM, "plan: sample table allocation or upload: %s",
                              cudaGetErrorString(cudaGetLastError())));
  *out = p;
  return DISORDER_OK;
}

int disorder_plan_destroy(disorder_plan p) {
  if (!p) return DISORDER_BAD_ARG;
  cudaSetDevice(p->ctx->device);
  cudaStreamSynchronize(p->ctx->stream);
  for (int m = 0; m < 3; ++m) {
    cudaFree(p->d_kG[m]);
    cudaFree(p->d_rG[m]);
    cudaFree(p->d_tw[m]);
  }
  cudaFree(p->d_ky);
  cudaFree(p->d_kz);
  cudaFree(p->d_seg_of);
  cudaFree(p->d_perm);
  cudaFree(p->d_kyq);
  cudaFree(p->d_kzq);
  cudaFree(p->d_rowptr);
  cudaFree(p->d_seg_off);
  delete p;
  return DISORDER_OK;
}

#define PLAN_CHECK(ctx, plan)                                                        \
  CTX_CHECK(ctx);                                                                    \
  if (!(plan) || (plan)->ctx != (ctx)) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan"); \
  DEV_GUARD(ctx)

static std::vector<int> all_segs(const disorder_plan_s* p) {
  std::vector<int> v(p->n_seg);
  std::iota(v.begin(), v.end(), 0);
  return v;
}

// ---------------------------------------------------------------- transform
int disorder_sinc_rigid_transform(disorder_ctx ctx, disorder_plan plan, const void* x, int32_t x_states,
                                  const float* T, int32_t n_states, int32_t di, int32_t sumR, int32_t useFull,
                                  void* out) {
  PLAN_CHECK(ctx, plan);
  if (!x || !T || !out || n_states < 1 || (x_states != 1 && x_states != n_states) || (di != 0 && di != 1) ||
      useFull < -1 || useFull > 1)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "sinc_rigid_transform: bad arguments");
  const long long V = plan->V;
  std::vector<SlotParams> prm;
  dis_slot_params(T, n_states, nullptr, n_states, di, &prm);
  const size_t tbytes = dis_table_bytes(plan, n_states, false);
  const bool need_copy = (di == 0 && sumR);
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, tbytes + (need_copy ? sizeof(float2) * V * n_states : 0) + (1 << 20), &ws));
  Tables tb;
  DIS_TRY(dis_build_tables(ctx, plan, prm, false, &ws, &tb));
  const float2* xin = (const float2*)x;
  if (di == 1) {
    DIS_TRY(dis_forward_transform(ctx, plan, xin, x_states == 1 ? 0 : V, (float2*)out, tb, useFull, nullptr));
    return DISORDER_OK;
  }
  float2* u = need_copy ? ws.take<float2>((size_t)V * n_states) : (float2*)out;
  if (!u) return dis_set_error(ctx, DISORDER_OOM, "workspace");
  if (x_states == 1 && n_states > 1) {
    DIS_TRY(dis_broadcast(ctx, xin, V, n_states, u));
  } else if ((const void*)u != x) {
    DIS_CUDA_TRY(cudaMemcpyAsync(u, xin, sizeof(float2) * V * n_states, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  DIS_TRY(dis_inverse_transform(ctx, plan, u, tb, useFull, sumR ? (float2*)out : nullptr, 0.f));
  return DISORDER_OK;
}

int disorder_sinc_rigid_transform_gradient(disorder_ctx ctx, disorder_plan plan, const void* x, const float* T,
                                           int32_t n_states, void* G, void* xT) {
  PLAN_CHECK(ctx, plan);
  if (!x || !T || !G || n_states < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "gradient: bad arguments");
  const long long V = plan->V;
  std::vector<SlotParams> prm;
  dis_slot_params(T, n_states, nullptr, n_states, 1, &prm);
  const size_t vols = (xT ? 4 : 5) * (size_t)n_states * V * sizeof(float2);
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, vols + dis_table_bytes(plan, n_states, true) + (1 << 20), &ws));
  Tables tb;
  DIS_TRY(dis_build_tables(ctx, plan, prm, true, &ws, &tb));
  float2* z = xT ? (float2*)xT : ws.take<float2>((size_t)n_states * V);
  float2* yB = ws.take<float2>((size_t)2 * n_states * V);
  float2* w1 = ws.take<float2>((size_t)n_states * V);
  float2* w2 = ws.take<float2>((size_t)n_states * V);
  if (!z || !yB || !w1 || !w2) return dis_set_error(ctx, DISORDER_OOM, "workspace");
  return dis_gradient(ctx, plan, (const float2*)x, 0, tb, z, yB, w1, w2, (float2*)G);
}

// ---------------------------------------------------------------- encoding
int disorder_encode(disorder_ctx ctx, disorder_plan plan, const void* x, const void* Sf, int32_t n_coils,
                    const float* T, void* y) {
  PLAN_CHECK(ctx, plan);
  if (!x || !Sf || !y || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "encode: bad arguments");
  EncodeSpec sp;
  sp.x = (const float2*)x;
  sp.Sf = (const float2*)Sf;
  sp.C = n_coils;
  sp.T = T;
  sp.T_n = plan->n_mot;
  sp.segs = all_segs(plan);
  sp.n3_lo = 0;
  sp.N3c = plan->N[2];
  sp.y_ld = plan->n_samples;
  sp.y_n3off = 0;
  sp.y_N3 = plan->N[2];
  return dis_encode_segments(ctx, plan, sp, (float2*)y, nullptr);
}

int disorder_decode(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf, int32_t n_coils,
                    const float* T, const float* We, const float* Mb, void* x) {
  PLAN_CHECK(ctx, plan);
  if (!x || !Sf || !y || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "decode: bad arguments");
  DecodeSpec sp;
  sp.y = (const float2*)y;
  sp.Sf = (const float2*)Sf;
  sp.C = n_coils;
  sp.T = T;
  sp.T_n = plan->n_mot;
  sp.segs = all_segs(plan);
  sp.We = We;
  sp.Mb = Mb;
  return dis_decode_segments(ctx, plan, sp, (float2*)x);
}

int disorder_encodedecode(disorder_ctx ctx, disorder_plan plan, const void* x, const void* Sf, int32_t n_coils,
                          const float* T, const float* We, void* out) {
  PLAN_CHECK(ctx, plan);
  if (!x || !Sf || !out || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "encodedecode: bad arguments");
  const long long wm = (long long)plan->n_seg * plan->N[0] * plan->N[1];
  Workspace ws;
  DIS_TRY(dis_workspace2(ctx, sizeof(float) * wm + (1 << 16), &ws));
  float* wmap = ws.take<float>(wm);
  if (!wmap) return dis_set_error(ctx, DISORDER_OOM, "workspace");
  DIS_TRY(dis_build_weight_map(ctx, plan, We, wmap, 1.f));
  EncodeDecodeSpec sp;
  sp.x = (const float2*)x;
  sp.Sf = (const float2*)Sf;
  sp.C = n_coils;
  sp.T = T;
  sp.T_n = plan->n_mot;
  sp.segs = all_segs(plan);
  sp.wmap = wmap;
  sp.We = We;
  return dis_encodedecode_segments(ctx, plan, sp, (float2*)out);
}

int disorder_compute_energy(disorder_ctx ctx, disorder_plan plan, const void* y, const void* x, const void* Sf,
                            int32_t n_coils, const float* T, const float* Mb, const float* Mbe, const float* R_Ti,
                            double* En) {
  PLAN_CHECK(ctx, plan);
  if (!x || !Sf || !y || !En || n_coils < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "energy: bad arguments");
  const long long ny = plan->n_samples * plan->N[2] * (long long)n_coils;
  Workspace ws;
  DIS_TRY(dis_workspace2(ctx, sizeof(float2) * ny + sizeof(float) * plan->N[2] + (1 << 16), &ws));
  float2* rbuf = ws.take<float2>(ny);
  float* roww = ws.take<float>(plan->N[2]);
  if (!rbuf || !roww) return dis_set_error(ctx, DISORDER_OOM, "workspace");
  const float* rw = nullptr;
  if (Mb || Mbe) {
    std::vector<float> a(plan->N[2], 1.f), b(plan->N[2], 1.f);
    if (Mb) DIS_CUDA_TRY(cudaMemcpy(a.data(), Mb, sizeof(float) * plan->N[2], cudaMemcpyDeviceToHost));
    if (Mbe) DIS_CUDA_TRY(cudaMemcpy(b.data(), Mbe, sizeof(float) * plan->N[2], cudaMemcpyDeviceToHost));
    for (int i = 0; i < plan->N[2]; ++i) a[i] *= b[i];
    DIS_CUDA_TRY(cudaMemcpy(roww, a.data(), sizeof(float) * plan->N[2], cudaMemcpyHostToDevice));
    rw = roww;
  }
  return dis_energy(ctx, plan, (const float2*)y, (const float2*)x, (const float2*)Sf, n_coils, T, rw, R_Ti, rbuf, En);
}

// ---------------------------------------------------------------- solvers
int disorder_cg_solve(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf, int32_t n_coils,
                      const float* T, const float* We, const float* Mb, const float* Mbe, const float* P_Se,
                      const float* C_Ma, const float* R_Ti, void* x_inout, int32_t x_init, int32_t nIt,
                      int32_t tolType, double tol, double* En, int32_t* n_en, int32_t* nn) {
  PLAN_CHECK(ctx, plan);
  if (!y || !Sf || !x_inout || n_coils < 1 || nIt < 0 || !n_en || !nn)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "cg_solve: bad arguments");
  CGSpec s;
  s.y = (const float2*)y;
  s.Sf = (const float2*)Sf;
  s.C = n_coils;
  s.T = T;
  s.We = We;
  s.Mb = Mb;
  s.Mbe = Mbe;
  s.P_Se = P_Se;
  s.C_Ma = C_Ma;
  s.R_Ti = R_Ti;
  int a = 0, b = 0;
  const int st = dis_cg_solve(ctx, plan, s, (float2*)x_inout, x_init, nIt, tolType, tol, En, &a, &b);
  *n_en = a;
  *nn = b;
  return st;
}

int disorder_cg_solve_residual(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf, int32_t n_coils,
                               const float* T, const float* We, const float* Mb, const float* Mbe, const float* P_Se,
                               const float* C_Ma, const float* R_Ti, void* x_inout, int32_t x_init, int32_t nIt,
                               int32_t tolType, double tol, double* En, int32_t* n_en, int32_t* nn, void* r_out) {
  PLAN_CHECK(ctx, plan);
  if (!y || !Sf || !x_inout || n_coils < 1 || nIt < 0 || !n_en || !nn || !r_out)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "cg_solve_residual: bad arguments");
  CGSpec s;
  s.y = (const float2*)y;
  s.Sf = (const float2*)Sf;
  s.C = n_coils;
  s.T = T;
  s.We = We;
  s.Mb = Mb;
  s.Mbe = Mbe;
  s.P_Se = P_Se;
  s.C_Ma = C_Ma;
  s.R_Ti = R_Ti;
  s.r_out = (float2*)r_out;
  int a = 0, b = 0;
  const int st = dis_cg_solve(ctx, plan, s, (float2*)x_inout, x_init, nIt, tolType, tol, En, &a, &b);
  *n_en = a;
  *nn = b;
  return st;
}

int disorder_lm_step(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf, int32_t n_coils,
                     const void* x, float* T, float* w, uint8_t* cT, float winit, const float* tL, int32_t n3_lo,
                     int32_t n3_hi, double* En, double* EnPrev) {
  PLAN_CHECK(ctx, plan);
  if (!y || !Sf || !x || !T || !w || !cT || !tL || n_coils < 1)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "lm_step: bad arguments");
  LMSpec s;
  s.y = (const float2*)y;
  s.Sf = (const float2*)Sf;
  s.C = n_coils;
  s.x = (const float2*)x;
  s.winit = winit;
  s.tL[0] = tL[0];
  s.tL[1] = tL[1];
  s.n3_lo = n3_lo;
  s.n3_hi = n3_hi;
  return dis_lm_step(ctx, plan, s, T, w, cT, En, EnPrev);
}

}  // extern "C"

int disorder_cg_solve_shearlet(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf, int32_t n_coils,
                               const float* T, const float* We, const float* Mb, const float* Mbe, const float* P_Se,
                               const float* C_Ma, const float* R_Ti, disorder_shearlet sh, const float* sh_We,
                               float sh_scale, void* x_inout, int32_t x_init, int32_t nIt, int32_t tolType,
                               double tol, double* En, int32_t* n_en, int32_t* nn) {
  PLAN_CHECK(ctx, plan);
  if (!y || !Sf || !x_inout || n_coils < 1 || nIt < 0 || !n_en || !nn || !sh || !sh_We)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "cg_solve_shearlet: bad arguments");
  if (dis_shearlet_ctx(sh) != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "cg_solve_shearlet: system of another context");
  int shN[3];
  dis_shearlet_size(sh, shN);
  for (int m = 0; m < 3; ++m)
    if (shN[m] != plan->N[m])
      return dis_set_error(ctx, DISORDER_BAD_ARG, "cg_solve_shearlet: shearlet size %d x %d x %d != plan size",
                           shN[0], shN[1], shN[2]);
  CGSpec s;
  s.y = (const float2*)y;
  s.Sf = (const float2*)Sf;
  s.C = n_coils;
  s.T = T;
  s.We = We;
  s.Mb = Mb;
  s.Mbe = Mbe;
  s.P_Se = P_Se;
  s.C_Ma = C_Ma;
  s.R_Ti = R_Ti;
  s.sh = sh;
  s.sh_We = sh_We;
  s.sh_scale = sh_scale;
  int a = 0, b = 0;
  const int st = dis_cg_solve(ctx, plan, s, (float2*)x_inout, x_init, nIt, tolType, tol, En, &a, &b);
  *n_en = a;
  *nn = b;
  return st;
}
