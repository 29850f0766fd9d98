// Encoding operators over the segments of a plan
// (Reconstruction/encode.m, decode.m, encodedecode.m; hot fields only).
// Segments are processed in chunks sized to the workspace budget; within a
// chunk every kernel covers all of the chunk's segments and coils.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "internal.h"
#include "encoding.h"

int dis_sum_slots(disorder_ctx_s* ctx, const float2* u, long long V, int n_slots, float2* out, float beta);
int dis_broadcast(disorder_ctx_s* ctx, const float2* x, long long V, int n_slots, float2* out);

size_t dis_budget_bytes() {
  const char* e = std::getenv("DISORDER_WORKSPACE_GB");
  double gb = e ? std::atof(e) : 24.0;
  if (gb < 0.25) gb = 0.25;
  return (size_t)(gb * (1ull << 30));
}

bool dis_any_motion(const float* T, int n) {
  if (!T) return false;
  for (int i = 0; i < 6 * n; ++i)
    if (T[i] != 0.f) return true;
  return false;
}

// table bytes for ns slots (upper bound)
size_t dis_table_bytes(const disorder_plan_s* plan, int ns, bool grad) {
  const long long N0 = plan->N[0], N1 = plan->N[1], N2 = plan->N[2];
  const long long shear = 2 * (N0 * N1 + N2 * N0 + N1 * N2);
  return (size_t)ns * (sizeof(float2) * (shear * (grad ? 2 : 1) + N0 + N1 + N2) + 15 * sizeof(double)) + 64 * 1024;
}

static CoilArgs coil_args(const disorder_plan_s* plan, const float2* Sf, int C, int n3_lo, int N3c, long long Vz,
                          int n_slots, const int* d_slot_seg) {
  CoilArgs a;
  a.N1 = plan->N[0];
  a.N2 = plan->N[1];
  a.N3c = N3c;
  a.Vz = Vz;
  a.Sf = Sf + (long long)n3_lo * plan->N[0] * plan->N[1];
  a.Sc = plan->V;
  a.C = C;
  a.n_slots = n_slots;
  a.d_slot_seg = d_slot_seg;
  return a;
}

int dis_upload_ints(disorder_ctx_s* ctx, Workspace* ws, const std::vector<int>& v, int** out) {
  *out = ws->take<int>(std::max<size_t>(v.size(), 1));
  if (!*out) return dis_set_error(ctx, DISORDER_OOM, "workspace too small");
  if (!v.empty())
    DIS_CUDA_TRY(cudaMemcpyAsync(*out, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  return DISORDER_OK;
}

// per-slot coil-stage bytes
static size_t coil_slot_bytes(const disorder_plan_s* plan, int C, int N3c) {
  return (size_t)C * plan->N[0] * plan->N[1] * N3c * sizeof(float2);
}

int dis_chunk_slots(const disorder_plan_s* plan, int C, int N3c, size_t extra_per_slot, int n_total) {
  const size_t per = coil_slot_bytes(plan, C, N3c) + extra_per_slot + dis_table_bytes(plan, 1, true);
  size_t budget = dis_budget_bytes();
  int ch = (int)std::max<size_t>(1, budget / std::max<size_t>(per, 1));
  return std::max(1, std::min(ch, n_total));
}

// ---------------------------------------------------------------- encode
int dis_encode_segments(disorder_ctx_s* ctx, const disorder_plan_s* plan, const EncodeSpec& sp, float2* y,
                        const float2* y_meas) {
  const long long V = plan->V;
  const int nsg = (int)sp.segs.size();
  if (nsg == 0) return DISORDER_OK;
  const bool motion = dis_any_motion(sp.T, sp.T_n);
  const int ch = dis_chunk_slots(plan, sp.C, sp.N3c, motion ? V * sizeof(float2) : 0, nsg);
  const size_t need = (size_t)ch * coil_slot_bytes(plan, sp.C, sp.N3c) + (motion ? (size_t)ch * V * sizeof(float2) : 0) +
                      dis_table_bytes(plan, ch, false) + 4096 * 4;
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, need, &ws));
  for (int c0 = 0; c0 < nsg; c0 += ch) {
    const int n = std::min(ch, nsg - c0);
    Workspace w = ws;
    std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
    float2* A = w.take<float2>((size_t)n * sp.C * plan->N[0] * plan->N[1] * sp.N3c);
    if (!A) return dis_set_error(ctx, DISORDER_OOM, "encode: workspace too small");
    const float2* z = sp.x;
    long long Vz = 0;
    if (motion) {
      float2* Z = w.take<float2>((size_t)n * V);
      if (!Z) return dis_set_error(ctx, DISORDER_OOM, "encode: workspace too small");
      std::vector<int> mot;
      for (int j = 0; j < n; ++j)
        if (segs[j] < plan->n_mot) mot.push_back(segs[j]);
      const int nm = (int)mot.size();  // motion segments come first in a chunk
      if (nm) {
        std::vector<SlotParams> prm;
        dis_slot_params(sp.T, sp.T_n, mot.data(), nm, 1, &prm);
        Tables tb;
        DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w, &tb));
        DIS_TRY(dis_forward_transform(ctx, plan, sp.x, 0, Z, tb, 1, nullptr));
      }
      if (n > nm) DIS_TRY(dis_broadcast(ctx, sp.x, V, n - nm, Z + (long long)nm * V));
      z = Z;
      Vz = V;
    }
    CoilArgs ca = coil_args(plan, sp.Sf, sp.C, sp.n3_lo, sp.N3c, Vz, n, d_seg);
    DIS_TRY(dis_coil_expand_fft1(ctx, plan, ca, z + (long long)sp.n3_lo * plan->N[0] * plan->N[1], A));
    const float scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
    DIS_TRY(dis_coil_fft2_gather(ctx, plan, ca, A, y, sp.y_ld, sp.y_n3off, sp.y_N3, y_meas, scale));
  }
  return DISORDER_OK;
}

// coil stage only, for per-slot volumes vols (stride V) whose segments are segs
int dis_encode_volumes(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* vols, const int* d_segs,
                       int n, const float2* Sf, int C, int n3_lo, int N3c, float2* A, float2* y, long long y_ld,
                       int y_n3off, int y_N3, const float2* y_meas) {
  CoilArgs ca = coil_args(plan, Sf, C, n3_lo, N3c, plan->V, n, d_segs);
  DIS_TRY(dis_coil_expand_fft1(ctx, plan, ca, vols + (long long)n3_lo * plan->N[0] * plan->N[1], A));
  const float scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
  return dis_coil_fft2_gather(ctx, plan, ca, A, y, y_ld, y_n3off, y_N3, y_meas, scale);
}

// ---------------------------------------------------------------- decode
int dis_decode_segments(disorder_ctx_s* ctx, const disorder_plan_s* plan, const DecodeSpec& sp, float2* out) {
  const long long V = plan->V;
  const int nsg = (int)sp.segs.size();
  if (nsg == 0) {
    DIS_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float2) * V, ctx->stream));
    return DISORDER_OK;
  }
  const bool motion = dis_any_motion(sp.T, sp.T_n);
  const int N3 = plan->N[2];
  const int ch = dis_chunk_slots(plan, sp.C, N3, V * sizeof(float2), nsg);
  const size_t need = (size_t)ch * (coil_slot_bytes(plan, sp.C, N3) + V * sizeof(float2)) +
                      dis_table_bytes(plan, ch, false) + 4096 * 4;
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, need, &ws));
  bool first = true;
  for (int c0 = 0; c0 < nsg; c0 += ch) {
    const int n = std::min(ch, nsg - c0);
    Workspace w = ws;
    std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
    float2* A = w.take<float2>((size_t)n * sp.C * V);
    float2* U = w.take<float2>((size_t)n * V);
    if (!A || !U) return dis_set_error(ctx, DISORDER_OOM, "decode: workspace too small");
    CoilArgs ca = coil_args(plan, sp.Sf, sp.C, 0, N3, V, n, d_seg);
    DIS_TRY(dis_coil_scatter_ifft2(ctx, plan, ca, sp.y, plan->n_samples, 0, N3, sp.We, sp.Mb, A));
    const float scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
    DIS_TRY(dis_coil_ifft1_combine(ctx, plan, ca, A, U, scale));
    int nm = 0;
    if (motion)
      for (int j = 0; j < n; ++j)
        if (segs[j] < plan->n_mot) ++nm;
    if (nm) {
      std::vector<SlotParams> prm;
      dis_slot_params(sp.T, sp.T_n, segs.data(), nm, 0, &prm);
      Tables tb;
      DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w, &tb));
      DIS_TRY(dis_inverse_transform(ctx, plan, U, tb, 1, out, first ? 0.f : 1.f));
      first = false;
    }
    if (n > nm) {
      DIS_TRY(dis_sum_slots(ctx, U + (long long)nm * V, V, n - nm, out, first ? 0.f : 1.f));
      first = false;
    }
  }
  return DISORDER_OK;
}

// ---------------------------------------------------------------- encodedecode
int dis_encodedecode_segments(disorder_ctx_s* ctx, const disorder_plan_s* plan, const EncodeDecodeSpec& sp,
                              float2* out) {
  const long long V = plan->V;
  const int nsg = (int)sp.segs.size();
  if (nsg == 0) {
    DIS_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float2) * V, ctx->stream));
    return DISORDER_OK;
  }
  const bool motion = dis_any_motion(sp.T, sp.T_n);
  const int N3 = plan->N[2];
  const int ch = dis_chunk_slots(plan, sp.C, N3, V * sizeof(float2), nsg);
  const size_t need = (size_t)ch * (coil_slot_bytes(plan, sp.C, N3) + V * sizeof(float2)) +
                      2 * dis_table_bytes(plan, ch, false) + 4096 * 4;
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, need, &ws));
  bool first = true;
  for (int c0 = 0; c0 < nsg; c0 += ch) {
    const int n = std::min(ch, nsg - c0);
    Workspace w = ws;
    std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
    float2* A = w.take<float2>((size_t)n * sp.C * V);
    float2* Z = w.take<float2>((size_t)n * V);
    if (!A || !Z) return dis_set_error(ctx, DISORDER_OOM, "encodedecode: workspace too small");
    int nm = 0;
    if (motion)
      for (int j = 0; j < n; ++j)
        if (segs[j] < plan->n_mot) ++nm;
    Tables tb;
    if (nm) {
      std::vector<SlotParams> prm;
      dis_slot_params(sp.T, sp.T_n, segs.data(), nm, 1, &prm);
      DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w, &tb));
      DIS_TRY(dis_forward_transform(ctx, plan, sp.x, 0, Z, tb, 1, nullptr));
    }
    const float2* z = Z;
    long long Vz = V;
    if (!motion) {
      z = sp.x;
      Vz = 0;
    } else if (n > nm) {
      DIS_TRY(dis_broadcast(ctx, sp.x, V, n - nm, Z + (long long)nm * V));
    }
    CoilArgs ca = coil_args(plan, sp.Sf, sp.C, 0, N3, Vz, n, d_seg);
    DIS_TRY(dis_coil_expand_fft1(ctx, plan, ca, z, A));
    DIS_TRY(dis_coil_fft2_weight(ctx, plan, ca, A, sp.wmap));
    ca.Vz = V;
    const float scale = (float)(1.0 / ((double)plan->N[0] * plan->N[1]));
    DIS_TRY(dis_coil_ifft1_combine(ctx, plan, ca, A, Z, scale));
    if (nm) {
      // inverse transform factors (di=0) for the motion slots
      std::vector<SlotParams> prm;
      dis_slot_params(sp.T, sp.T_n, segs.data(), nm, 0, &prm);
      Tables tbi;
      DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w, &tbi));
      DIS_TRY(dis_inverse_transform(ctx, plan, Z, tbi, 1, out, first ? 0.f : 1.f));
      first = false;
    }
    if (n > nm) {
      DIS_TRY(dis_sum_slots(ctx, Z + (long long)nm * V, V, n - nm, out, first ? 0.f : 1.f));
      first = false;
    }
  }
  return DISORDER_OK;
}
