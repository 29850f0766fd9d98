// Sinc rigid transform that allocates nothing.
//
// disorder_sinc_rigid_transform builds its per-state phase tables in the
// context's workspace, which the library grows with cudaMalloc on demand. Some
// callers cannot let a library allocate device memory in the middle of their
// pipeline: a scanner's online reconstruction host or another application that
// reserves its whole device-memory budget at start-up and hands buffers out
// from its own allocator, where a cudaMalloc can fail once that budget is
// taken and, besides, synchronises the device. For them this entry point keeps
// all of its scratch (the phase tables and the per-state scalars) in one
// file-scope device array of fixed size, kStaticScratchBytes (32 MiB).
//
// The array's device address is resolved once per context, when the context
// is created (dis_static_scratch_resolve, called by disorder_ctx_create with
// the context's device current). That first cudaGetSymbolAddress also loads
// the module holding the array, which commits its 32 MiB on that device; the
// device keeps them until the process exits. The entry point itself then
// makes no allocation and loads no data module.
#include <cstring>

#include "internal.h"

namespace {

constexpr size_t kStaticScratchBytes = 32ull << 20;
__device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

}  // namespace

// In host code g_scratch names a host-side stand-in, not device memory: a
// kernel handed it would fault or read the wrong memory. The runtime gives the
// array's address on the current device.
int dis_static_scratch_resolve(void** addr, size_t* bytes) {
  *addr = nullptr;
  *bytes = 0;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return DISORDER_CUDA_ERR;
  }
  *addr = p;
  *bytes = kStaticScratchBytes;
  return DISORDER_OK;
}

extern "C" int disorder_sinc_rigid_transform_static(disorder_ctx ctx, disorder_plan plan, const void* x,
                                                    int32_t x_states, const float* T, int32_t n_states, int32_t di,
                                                    int32_t useFull, void* out) {
  if (!ctx) return DISORDER_BAD_ARG;
  if (!plan || plan->ctx != ctx) return dis_set_error(ctx, DISORDER_BAD_ARG, "bad plan");
  if (!x || !T || !out || n_states < 1 || (di != 0 && di != 1) || useFull < -1 || useFull > 1)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "sinc_rigid_transform_static: bad arguments");
  if (di == 1 && x_states != 1 && x_states != n_states)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "sinc_rigid_transform_static: x_states must be 1 or n_states");
  if (di == 0 && x_states != n_states)
    return dis_set_error(ctx, DISORDER_BAD_ARG,
                         "sinc_rigid_transform_static: the inverse takes n_states volumes and does not sum them");
  if (n_states > kMaxStaticSlots)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "sinc_rigid_transform_static: at most %d states per call",
                         kMaxStaticSlots);
  const size_t need = dis_static_table_bytes(plan, n_states);
  if (need > kStaticScratchBytes)
    return dis_set_error(ctx, DISORDER_BAD_ARG,
                         "sinc_rigid_transform_static: %d states of a %dx%dx%d grid need %zu bytes of scratch; "
                         "the static scratch holds %zu bytes (use fewer states per call)",
                         n_states, plan->N[0], plan->N[1], plan->N[2], need, kStaticScratchBytes);
  if (!ctx->static_scratch)
    return dis_set_error(ctx, DISORDER_CUDA_ERR,
                         "sinc_rigid_transform_static: the static scratch address could not be resolved when the "
                         "context was created");
  // per-state scalars staged in thread-local static storage: no heap, and no
  // large stack frame on the caller's thread
  static thread_local SlotParams sp[kMaxStaticSlots];
  dis_slot_params_into(T, n_states, di, sp);
  for (int s = 0; s < n_states; ++s)
    if (sp[s].flip[0] || sp[s].flip[1] || sp[s].flip[2])
      return dis_set_error(ctx, DISORDER_BAD_ARG,
                           "sinc_rigid_transform_static: rotations beyond 90 degrees are not supported here "
                           "(state %d); use disorder_sinc_rigid_transform",
                           s);
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  Tables tb;
  const int st = dis_build_tables_into(ctx, plan, sp, n_states, (char*)ctx->static_scratch,
                                       ctx->static_scratch_bytes, &tb);
  if (st == DISORDER_OOM)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "sinc_rigid_transform_static: tables exceed the static scratch");
  if (st != DISORDER_OK) return st;
  const long long V = plan->V;
  if (di == 1) return dis_forward_transform(ctx, plan, (const float2*)x, x_states == 1 ? 0 : V, (float2*)out, tb,
                                            useFull, nullptr);
  if (out != x)
    DIS_CUDA_TRY(cudaMemcpyAsync(out, x, sizeof(float2) * V * n_states, cudaMemcpyDeviceToDevice, ctx->stream));
  return dis_inverse_transform(ctx, plan, (float2*)out, tb, useFull, nullptr, 0.f);
}
