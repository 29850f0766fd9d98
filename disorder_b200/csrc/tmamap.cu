// Tensor maps and size dispatch of the TMA line passes (tmapass.cuh).
#include <cudaTypedefs.h>

#include <cstdlib>

#include "fastpass.h"
#include "internal.h"
#include "tmapass.cuh"

extern template struct fp::TmaLaunch<4, 11>;
extern template struct fp::TmaLaunch<8, 11>;
extern template struct fp::TmaLaunch<8, 12>;
extern template struct fp::TmaLaunch<16, 8>;
extern template struct fp::TmaLaunch<16, 10>;
extern template struct fp::TmaLaunch<16, 11>;
extern template struct fp::TmaLaunch<16, 12>;
extern template struct fp::TmaLaunch<16, 16>;

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

bool tma_enabled() {
  static const bool v = [] {
    const char* e = std::getenv("DISORDER_NO_TMA");
    return !(e && e[0] == '1');
  }();
  return v;
}

bool launch_size(int n, int kind, const CUtensorMap& in, const CUtensorMap& out, const fp::TArgs& t,
                 const float2* tw, int shared_input, cudaStream_t s) {
  switch (n) {
    case 44: return fp::TmaLaunch<4, 11>::launch(kind, in, out, t, tw, shared_input, s);
    case 88: return fp::TmaLaunch<8, 11>::launch(kind, in, out, t, tw, shared_input, s);
    case 96: return fp::TmaLaunch<8, 12>::launch(kind, in, out, t, tw, shared_input, s);
    case 128: return fp::TmaLaunch<16, 8>::launch(kind, in, out, t, tw, shared_input, s);
    case 160: return fp::TmaLaunch<16, 10>::launch(kind, in, out, t, tw, shared_input, s);
    case 176: return fp::TmaLaunch<16, 11>::launch(kind, in, out, t, tw, shared_input, s);
    case 192: return fp::TmaLaunch<16, 12>::launch(kind, in, out, t, tw, shared_input, s);
    case 256: return fp::TmaLaunch<16, 16>::launch(kind, in, out, t, tw, shared_input, s);
    default: return false;
  }
}

bool has_tma_size(int n) {
  switch (n) {
    case 44: case 88: case 96: case 128: case 160: case 176: case 192: case 256: return true;
    default: return false;
  }
}

}  // namespace

bool dis_tmap_volumes(CUtensorMap* m, const void* base, const int* N, int axis, long long vol_stride, int n_vol) {
  auto enc = encode_fn();
  if (!enc || (axis != 1 && axis != 2)) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (N[0] & 1) || n_vol < 1) return false;
  const long long V = (long long)N[0] * N[1] * N[2];
  if (n_vol == 1) vol_stride = V;  // unused dimension: any stride that follows the rules
  if (vol_stride < V || (vol_stride & 1)) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)N[0], (cuuint64_t)N[1], (cuuint64_t)N[2], (cuuint64_t)n_vol};
  const cuuint64_t strides[3] = {(cuuint64_t)N[0] * 8, (cuuint64_t)N[0] * N[1] * 8, (cuuint64_t)vol_stride * 8};
  const cuuint32_t box[4] = {16, axis == 1 ? (cuuint32_t)N[1] : 1u, axis == 2 ? (cuuint32_t)N[2] : 1u, 1};
  if (box[1] > 256 || box[2] > 256) return false;
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, const_cast<void*>(base), dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// an injected wait fault (disorder_ctx_inject_fault) applies to the next
// TMA pass only
static void take_fault(disorder_ctx_s* ctx, fp::TArgs& t) {
  if (ctx->fault == DISORDER_FAULT_TMA_WAIT) {
    ctx->fault = DISORDER_FAULT_NONE;
    t.skip_loads = 1;
    t.wait_limit = 1u << 12;
  }
}

bool dis_umma_line(int n, int mode, const CUtensorMap& in, const CUtensorMap& out, const fp::TArgs& t,
                   const float2* tw, int shared_input, int sm_count, cudaStream_t s);

bool dis_fast_tma_line(disorder_ctx_s* ctx, const LinePassArgs& a) {
  if (!tma_enabled() || !ctx->tune_tma || !ctx->d_err) return false;
  if (a.axis == 0 || a.accumulate || a.in1 || a.out1 || a.c01 != P_ZERO) return false;
  if (!a.Sd.p || !(a.c00 == P_A || a.c00 == P_ONE)) return false;
  const int n = a.N[a.axis];
  if (!has_tma_size(n)) return false;
  int F1, F2;
  if (!dis_fast_factor(n, &F1, &F2) || a.sd_w != 2 * F1 + 2) return false;
  const int shared_input = a.in0_s == 0 ? 1 : 0;
  CUtensorMap in, out;
  if (!dis_tmap_volumes(&in, a.in0, a.N, a.axis, a.in0_s, shared_input ? 1 : a.n_slots)) return false;
  if (!dis_tmap_volumes(&out, a.out0, a.N, a.axis, a.out0_s, a.n_slots)) return false;
  fp::TArgs t;
  for (int i = 0; i < 3; ++i) t.Nv[i] = a.N[i];
  t.axis = a.axis;
  t.n_vol = a.n_slots;
  t.n_slots = a.n_slots;
  t.C = 1;
  t.slot_seg = nullptr;
  t.wmap = nullptr;
  t.a = a;
  t.err = ctx->d_err;
  take_fault(ctx, t);
  // mixed precision: the DFTs of the pass as tensor-core GEMMs where a kernel exists
  if (ctx->precision != DISORDER_PRECISION_FP32 && F1 == 16 &&
      dis_umma_line(n, ctx->precision, in, out, t, a.tw, shared_input, ctx->sm_count, ctx->stream))
    return true;
  return launch_size(n, 0, in, out, t, a.tw, shared_input, ctx->stream);
}

bool dis_fast_tma_weight(disorder_ctx_s* ctx, const CoilArgs& a, float2* A, const float* wmap, const float2* tw,
                         const disorder_plan_s* plan, float2* ys, long long ld, int n3off, int N3y, float scale) {
  if (!tma_enabled() || !ctx->tune_tma || !ctx->d_err || !has_tma_size(a.N2)) return false;
  const int Nv[3] = {a.N1, a.N2, a.N3c};
  const long long Vc = (long long)a.N1 * a.N2 * a.N3c;
  const long long nvol = (long long)a.n_slots * a.C;
  if (nvol < 1 || nvol >= (1LL << 31)) return false;
  CUtensorMap m;
  if (!dis_tmap_volumes(&m, A, Nv, 1, Vc, (int)nvol)) return false;
  fp::TArgs t = fp::TArgs();
  for (int i = 0; i < 3; ++i) t.Nv[i] = Nv[i];
  t.axis = 1;
  t.n_vol = (int)nvol;
  t.n_slots = a.n_slots;
  t.C = a.C;
  t.slot_seg = a.d_slot_seg;
  t.wmap = wmap;
  t.err = ctx->d_err;
  if (ys) {
    t.y = ys;
    t.ld = ld;
    t.n3off = n3off;
    t.N3y = N3y;
    t.scale = scale;
    t.rowptr = plan->d_rowptr;
    t.perm = plan->d_perm;
    t.kyv = plan->d_ky;
    t.kzv = plan->d_kz;
  }
  take_fault(ctx, t);
  return launch_size(a.N2, 1, m, m, t, tw, 0, ctx->stream);
}

namespace {
bool coil_tma(disorder_ctx_s* ctx, int kind, const CoilArgs& a, float2* A, const disorder_plan_s* plan,
              fp::TArgs& t) {
  if (!tma_enabled() || !ctx->tune_tma || !ctx->d_err || !has_tma_size(a.N2)) return false;
  const int Nv[3] = {a.N1, a.N2, a.N3c};
  const long long Vc = (long long)a.N1 * a.N2 * a.N3c;
  const long long nvol = (long long)a.n_slots * a.C;
  if (nvol < 1 || nvol >= (1LL << 31)) return false;
  CUtensorMap m;
  if (!dis_tmap_volumes(&m, A, Nv, 1, Vc, (int)nvol)) return false;
  for (int i = 0; i < 3; ++i) t.Nv[i] = Nv[i];
  t.axis = 1;
  t.n_vol = (int)nvol;
  t.n_slots = a.n_slots;
  t.C = a.C;
  t.slot_seg = a.d_slot_seg;
  t.err = ctx->d_err;
  t.rowptr = plan->d_rowptr;
  t.perm = plan->d_perm;
  t.kyv = plan->d_ky;
  t.kzv = plan->d_kz;
  take_fault(ctx, t);
  return launch_size(a.N2, kind, m, m, t, plan->d_tw[1], 0, ctx->stream);
}
}  // namespace

bool dis_fast_tma_gather(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* A,
                         float2* y, long long y_ld, int y_n3off, int y_N3, const float2* y_meas, float scale) {
  fp::TArgs t = fp::TArgs();
  t.y = y;
  t.ymeas = y_meas;
  t.ld = y_ld;
  t.n3off = y_n3off;
  t.N3y = y_N3;
  t.scale = scale;
  return coil_tma(ctx, 2, a, const_cast<float2*>(A), plan, t);
}

bool dis_fast_tma_scatter(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* y,
                          long long y_ld, int y_n3off, int y_N3, const float* We, const float* Mb, float2* A) {
  fp::TArgs t = fp::TArgs();
  t.y = const_cast<float2*>(y);
  t.ld = y_ld;
  t.n3off = y_n3off;
  t.N3y = y_N3;
  t.We = We;
  t.Mb = Mb;
  return coil_tma(ctx, 3, a, A, plan, t);
}
