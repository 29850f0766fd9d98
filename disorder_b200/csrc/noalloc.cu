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
// file-scope device array of fixed size, kStaticScratchBytes (32 MiB), that
// every GPU which loads this library holds until the process exits.
#include <cstring>

#include "internal.h"

namespace {

constexpr size_t kStaticScratchBytes = 32ull << 20;
__device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {};

// bytes the tables of n states need in the static scratch (with the 256-byte
// rounding of every sub-allocation)
size_t table_bytes(const disorder_plan_s* p, int n) {
  auto r = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t N0 = p->N[0], N1 = p->N[1], N2 = p->N[2];
  size_t b = r(15 * sizeof(double) * n);
  b += 2 * (r(sizeof(float2) * N0 * N1 * n) + r(sizeof(float2) * N2 * N0 * n) + r(sizeof(float2) * N1 * N2 * n));
  b += r(sizeof(float2) * N0 * n) + r(sizeof(float2) * N1 * n) + r(sizeof(float2) * N2 * n);
  return b;
}

}  // namespace

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
  const size_t need = table_bytes(plan, n_states);
  if (need > kStaticScratchBytes)
    return dis_set_error(ctx, DISORDER_BAD_ARG,
                         "sinc_rigid_transform_static: %d states of a %dx%dx%d grid need %zu bytes of scratch; "
                         "the static scratch holds %zu bytes (use fewer states per call)",
                         n_states, plan->N[0], plan->N[1], plan->N[2], need, kStaticScratchBytes);
  SlotParams sp[kMaxStaticSlots];
  dis_slot_params_into(T, n_states, di, sp);
  for (int s = 0; s < n_states; ++s)
    if (sp[s].flip[0] || sp[s].flip[1] || sp[s].flip[2])
      return dis_set_error(ctx, DISORDER_BAD_ARG,
                           "sinc_rigid_transform_static: rotations beyond 90 degrees are not supported here "
                           "(state %d); use disorder_sinc_rigid_transform",
                           s);
  DIS_CUDA_TRY(cudaSetDevice(ctx->device));
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return dis_set_error(ctx, DISORDER_BAD_ARG, "sinc_rigid_transform_static: device %d", ctx->device);
  // set-up, once per device and with that device current: the host-side name
  // g_scratch is not a device address, so take the address from the runtime
  if (!g_scratch_addr[ctx->device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      return dis_set_error(ctx, DISORDER_CUDA_ERR, "cudaGetSymbolAddress(static scratch): %s", cudaGetErrorString(e));
    g_scratch_addr[ctx->device] = p;
  }
  Tables tb;
  const int st = dis_build_tables_into(ctx, plan, sp, n_states, (char*)g_scratch_addr[ctx->device],
                                       kStaticScratchBytes, &tb);
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
