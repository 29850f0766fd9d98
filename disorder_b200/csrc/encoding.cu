// Encoding operators over the segments of a plan
// (Reconstruction/encode.m, decode.m, encodedecode.m; hot fields only).
// The coil stage runs as the fused plane kernel (plane.cuh) when its shared
// memory fits (C x samples-per-segment); otherwise as three passes through
// per-coil buffers (coil.cu). Segments are processed in chunks sized to the
// workspace budget.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "encoding.h"
#include "fastpass.h"
#include "internal.h"
#include "plane.cuh"

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
  const long long seeds = 34 * (3 * (N0 + N1 + N2) + 3);  // rows of at most 2*16+2 seeds
  return (size_t)ns * (sizeof(float2) * (shear * (grad ? 2 : 1) + N0 + N1 + N2 + seeds) + 15 * sizeof(double)) +
         64 * 1024;
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

// per-slot coil-stage bytes of the three-pass path
static size_t coil_slot_bytes(const disorder_plan_s* plan, int C, int N3c) {
  return (size_t)C * plan->N[0] * plan->N[1] * N3c * sizeof(float2);
}

// most samples of any of the segments
static int max_samples(const disorder_plan_s* plan, const std::vector<int>& segs);

// The coil stage of a call: the sample-sum stage (sumcoil.cu) when it has a
// kernel for the sizes and its partial sums per slot are no larger than the
// three-pass stage's per-coil volumes (at most N1 x lines-per-CTA samples per
// segment), else the three passes. ldp: the partial sums' sample stride.
struct CoilPlan {
  bool sum = false;
  int ldp = 0;
  size_t per_slot = 0;  // coil-stage workspace bytes per slot
  size_t gather = 0;    // sample-sum adjoint: its gathered samples per slot
};
static CoilPlan coil_plan(const disorder_plan_s* plan, int C, int N3c, const std::vector<int>& segs) {
  CoilPlan p;
  p.per_slot = coil_slot_bytes(plan, C, N3c);
  if (!dis_sum_coil_usable(plan)) return p;
  const int ldp = std::max(1, max_samples(plan, segs));
  const size_t pb = dis_sum_part_bytes(plan, C, N3c, ldp);
  if (pb > p.per_slot) return p;
  p.sum = true;
  p.ldp = ldp;
  p.per_slot = pb;
  p.gather = dis_sum_gather_bytes(C, N3c, ldp);
  return p;
}

// slots per chunk for a coil stage of coil bytes per slot and extra bytes per slot
static int chunk_for(const disorder_plan_s* plan, size_t coil, size_t extra, int n_total) {
  const size_t per = coil + extra + dis_table_bytes(plan, 1, true);
  const int ch = (int)std::max<size_t>(1, dis_budget_bytes() / std::max<size_t>(per, 1));
  return std::max(1, std::min(ch, n_total));
}

int dis_chunk_slots(const disorder_plan_s* plan, int C, int N3c, size_t extra_per_slot, int n_total) {
  const size_t per = coil_slot_bytes(plan, C, N3c) + extra_per_slot + dis_table_bytes(plan, 1, true);
  size_t budget = dis_budget_bytes();
  int ch = (int)std::max<size_t>(1, budget / std::max<size_t>(per, 1));
  return std::max(1, std::min(ch, n_total));
}

// ---------------------------------------------------------------- plane path
static int max_samples(const disorder_plan_s* plan, const std::vector<int>& segs) {
  long long m = 0;
  for (int s : segs) m = std::max(m, plan->seg_off[s + 1] - plan->seg_off[s]);
  return (int)m;
}

// The fused plane kernel trades HBM traffic for arithmetic (the restricted
// DFT costs Ns*N2 MACs per coil-plane) and holds one CTA per SM at 256x256;
// on B200 the three-pass path is faster at the benchmark sizes, so the plane
// kernel is used only when DISORDER_PLANE=1.
static bool plane_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = std::getenv("DISORDER_PLANE");
    v = (e && e[0] == '1') ? 1 : 0;
  }
  return v == 1;
}

bool dis_plane_usable(const disorder_plan_s* plan, int C, const std::vector<int>& segs) {
  if (!dis_use_fast() || !plane_enabled()) return false;
  const size_t b = dis_plane_smem(plan->N[0], plan->N[1], C, std::max(1, max_samples(plan, segs)));
  return b <= 225 * 1024;
}

static int plane_run(disorder_ctx_s* ctx, const disorder_plan_s* plan, int mode, const float2* z, long long Vz,
                     float2* u, long long Vu, const float2* Sf, int C, int n3_lo, int N3c, const int* d_seg, int n_slots,
                     int max_ns, float2* y, const float2* ymeas, long long ld, int y_n3off, int y_N3,
                     const float* We, const float* Mb) {
  if (n_slots == 0 || N3c == 0) return DISORDER_OK;
  const long long pl3 = (long long)n3_lo * plan->N[0] * plan->N[1];
  pl::PlaneArgs a;
  a.N1 = plan->N[0];
  a.N2 = plan->N[1];
  a.N3c = N3c;
  a.Vz = Vz;
  a.Vu = Vu;
  a.z = z + pl3;
  a.u = u ? u + pl3 : nullptr;
  a.Sf = Sf + pl3;
  a.Sc = plan->V;
  a.C = C;
  a.slot_seg = d_seg;
  a.seg_off = plan->d_seg_off;
  a.ky = plan->d_ky;
  a.kz = plan->d_kz;
  a.rowptr = plan->d_rowptr;
  a.perm = plan->d_perm;
  a.y = y;
  a.ymeas = ymeas;
  a.ld = ld;
  a.y_n3off = y_n3off;
  a.y_N3 = y_N3;
  a.We = We;
  a.Mb = Mb;
  const double n12 = (double)plan->N[0] * plan->N[1];
  a.scale_f = (float)(1.0 / std::sqrt(n12));
  a.scale_a = (float)(mode == pl::ENCDEC ? 1.0 / n12 : 1.0 / std::sqrt(n12));
  a.max_ns = std::max(1, max_ns);
  if (!dis_fast_plane(plan->N[0], mode, a, plan->d_tw[0], plan->d_tw[1], n_slots, ctx->stream))
    return dis_set_error(ctx, DISORDER_BAD_ARG, "plane kernel unavailable for N1=%d", plan->N[0]);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

// forward transform of the chunk's motion segments into Z, untransformed
// copies for the outer segments; returns the state volumes and their stride
static int states_of(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* x, const float* T, int T_n,
                     bool motion, const std::vector<int>& segs, Workspace* w, const float2** z, long long* Vz,
                     float2** Zout, int* n_mot) {
  const long long V = plan->V;
  const int n = (int)segs.size();
  *n_mot = 0;
  if (!motion) {
    *z = x;
    *Vz = 0;
    if (Zout) *Zout = nullptr;
    return DISORDER_OK;
  }
  float2* Z = w->take<float2>((size_t)n * V);
  if (!Z) return dis_set_error(ctx, DISORDER_OOM, "workspace too small");
  std::vector<int> mot;
  for (int s : segs)
    if (s < plan->n_mot) mot.push_back(s);
  const int nm = (int)mot.size();  // motion segments come first
  if (nm) {
    std::vector<SlotParams> prm;
    dis_slot_params(T, T_n, mot.data(), nm, 1, &prm);
    Tables tb;
    DIS_TRY(dis_build_tables(ctx, plan, prm, false, w, &tb));
    DIS_TRY(dis_forward_transform(ctx, plan, x, 0, Z, tb, 1, nullptr));
  }
  if (n > nm) DIS_TRY(dis_broadcast(ctx, x, V, n - nm, Z + (long long)nm * V));
  *z = Z;
  *Vz = V;
  if (Zout) *Zout = Z;
  *n_mot = nm;
  return DISORDER_OK;
}

// inverse transform of the motion slots of U summed into out, outer slots added
static int sum_back(disorder_ctx_s* ctx, const disorder_plan_s* plan, float2* U, const float* T, int T_n,
                    const std::vector<int>& segs, int nm, Workspace* w, float2* out, bool* first) {
  const long long V = plan->V;
  const int n = (int)segs.size();
  if (nm) {
    std::vector<SlotParams> prm;
    dis_slot_params(T, T_n, segs.data(), nm, 0, &prm);
    Tables tb;
    DIS_TRY(dis_build_tables(ctx, plan, prm, false, w, &tb));
    DIS_TRY(dis_inverse_transform(ctx, plan, U, tb, 1, out, *first ? 0.f : 1.f));
    *first = false;
  }
  if (n > nm) {
    DIS_TRY(dis_sum_slots(ctx, U + (long long)nm * V, V, n - nm, out, *first ? 0.f : 1.f));
    *first = false;
  }
  return DISORDER_OK;
}

static int plane_chunk(const disorder_plan_s* plan, int nsg, size_t per_slot) {
  const size_t per = per_slot + dis_table_bytes(plan, 1, false);
  const int ch = (int)std::max<size_t>(1, dis_budget_bytes() / std::max<size_t>(per, 1));
  return std::max(1, std::min(ch, nsg));
}

// ---------------------------------------------------------------- encode
int dis_encode_segments(disorder_ctx_s* ctx, const disorder_plan_s* plan, const EncodeSpec& sp, float2* y,
                        const float2* y_meas) {
  const long long V = plan->V;
  const int nsg = (int)sp.segs.size();
  if (nsg == 0) return DISORDER_OK;
  const bool motion = dis_any_motion(sp.T, sp.T_n);
  if (dis_plane_usable(plan, sp.C, sp.segs)) {
    const int ch = motion ? plane_chunk(plan, nsg, V * sizeof(float2)) : nsg;
    Workspace ws;
    DIS_TRY(dis_workspace(ctx, (motion ? (size_t)ch * V * sizeof(float2) : 0) + dis_table_bytes(plan, ch, false) +
                                   (1 << 20), &ws));
    for (int c0 = 0; c0 < nsg; c0 += ch) {
      const int n = std::min(ch, nsg - c0);
      Workspace w = ws;
      std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
      int* d_seg = nullptr;
      DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
      const float2* z;
      long long Vz;
      int nm;
      DIS_TRY(states_of(ctx, plan, sp.x, sp.T, sp.T_n, motion, segs, &w, &z, &Vz, nullptr, &nm));
      DIS_TRY(plane_run(ctx, plan, pl::ENCODE, z, Vz, nullptr, 0, sp.Sf, sp.C, sp.n3_lo, sp.N3c, d_seg, n,
                        max_samples(plan, segs), y, y_meas, sp.y_ld, sp.y_n3off, sp.y_N3, nullptr, nullptr));
    }
    return DISORDER_OK;
  }
  const CoilPlan cp = coil_plan(plan, sp.C, sp.N3c, sp.segs);
  const int ch = chunk_for(plan, cp.per_slot, motion ? V * sizeof(float2) : 0, nsg);
  const size_t need = (size_t)ch * cp.per_slot + (motion ? (size_t)ch * V * sizeof(float2) : 0) +
                      dis_table_bytes(plan, ch, false) + 4096 * 4;
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, need, &ws));
  for (int c0 = 0; c0 < nsg; c0 += ch) {
    const int n = std::min(ch, nsg - c0);
    Workspace w = ws;
    std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
    float2* A = w.take<float2>((size_t)n * cp.per_slot / sizeof(float2));
    if (!A) return dis_set_error(ctx, DISORDER_OOM, "encode: workspace too small");
    const float2* z;
    long long Vz;
    int nm;
    DIS_TRY(states_of(ctx, plan, sp.x, sp.T, sp.T_n, motion, segs, &w, &z, &Vz, nullptr, &nm));
    CoilArgs ca = coil_args(plan, sp.Sf, sp.C, sp.n3_lo, sp.N3c, Vz, n, d_seg);
    const float scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
    const float2* z3 = z + (long long)sp.n3_lo * plan->N[0] * plan->N[1];
    if (cp.sum) {
      DIS_TRY(dis_coil_sum_fwd(ctx, plan, ca, z3, A, cp.ldp, y, sp.y_ld, sp.y_n3off, sp.y_N3, y_meas, scale));
    } else {
      DIS_TRY(dis_coil_expand_fft1(ctx, plan, ca, z3, A));
      DIS_TRY(dis_coil_fft2_gather(ctx, plan, ca, A, y, sp.y_ld, sp.y_n3off, sp.y_N3, y_meas, scale));
    }
  }
  return DISORDER_OK;
}

// coil stage only, for per-slot volumes vols (stride V) whose segments are segs
int dis_encode_volumes(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* vols, const int* d_segs,
                       const std::vector<int>& segs, const float2* Sf, int C, int n3_lo, int N3c, float2* A,
                       float2* y, long long y_ld, int y_n3off, int y_N3, const float2* y_meas) {
  const int n = (int)segs.size();
  if (dis_plane_usable(plan, C, segs))
    return plane_run(ctx, plan, pl::ENCODE, vols, plan->V, nullptr, 0, Sf, C, n3_lo, N3c, d_segs, n,
                     max_samples(plan, segs), y, y_meas, y_ld, y_n3off, y_N3, nullptr, nullptr);
  if (!A) return dis_set_error(ctx, DISORDER_OOM, "encode_volumes: no coil buffer");
  CoilArgs ca = coil_args(plan, Sf, C, n3_lo, N3c, plan->V, n, d_segs);
  const float scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
  const float2* v3 = vols + (long long)n3_lo * plan->N[0] * plan->N[1];
  // A holds the three-pass stage's per-coil volumes; the sample-sum stage's
  // partial sums are never larger (coil_plan)
  const CoilPlan cp = coil_plan(plan, C, N3c, segs);
  if (cp.sum) return dis_coil_sum_fwd(ctx, plan, ca, v3, A, cp.ldp, y, y_ld, y_n3off, y_N3, y_meas, scale);
  DIS_TRY(dis_coil_expand_fft1(ctx, plan, ca, v3, A));
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
  bool first = true;
  if (dis_plane_usable(plan, sp.C, sp.segs)) {
    const int ch = plane_chunk(plan, nsg, V * sizeof(float2));
    Workspace ws;
    DIS_TRY(dis_workspace(ctx, (size_t)ch * V * sizeof(float2) + dis_table_bytes(plan, ch, false) + (1 << 20), &ws));
    for (int c0 = 0; c0 < nsg; c0 += ch) {
      const int n = std::min(ch, nsg - c0);
      Workspace w = ws;
      std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
      int* d_seg = nullptr;
      DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
      float2* U = w.take<float2>((size_t)n * V);
      if (!U) return dis_set_error(ctx, DISORDER_OOM, "decode: workspace too small");
      DIS_TRY(plane_run(ctx, plan, pl::DECODE, U, V, U, V, sp.Sf, sp.C, 0, N3, d_seg, n, max_samples(plan, segs),
                        const_cast<float2*>(sp.y), nullptr, plan->n_samples, 0, N3, sp.We, sp.Mb));
      int nm = 0;
      if (motion)
        for (int s : segs)
          if (s < plan->n_mot) ++nm;
      DIS_TRY(sum_back(ctx, plan, U, sp.T, sp.T_n, segs, nm, &w, out, &first));
    }
    return DISORDER_OK;
  }
  const CoilPlan cp = coil_plan(plan, sp.C, N3, sp.segs);
  const size_t coil = cp.sum ? cp.gather : cp.per_slot;
  const int ch = chunk_for(plan, coil, V * sizeof(float2), nsg);
  const size_t need = (size_t)ch * (coil + V * sizeof(float2)) + dis_table_bytes(plan, ch, false) + 4096 * 4;
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, need, &ws));
  for (int c0 = 0; c0 < nsg; c0 += ch) {
    const int n = std::min(ch, nsg - c0);
    Workspace w = ws;
    std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
    float2* A = w.take<float2>((size_t)n * (cp.sum ? cp.gather / sizeof(float2) : (size_t)sp.C * V));
    float2* U = w.take<float2>((size_t)n * V);
    if (!A || !U) return dis_set_error(ctx, DISORDER_OOM, "decode: workspace too small");
    CoilArgs ca = coil_args(plan, sp.Sf, sp.C, 0, N3, V, n, d_seg);
    const float scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
    if (cp.sum) {
      DIS_TRY(dis_coil_sum_adj(ctx, plan, ca, sp.y, plan->n_samples, 0, N3, sp.We, sp.Mb, U, scale, A, cp.ldp));
    } else {
      DIS_TRY(dis_coil_scatter_ifft2(ctx, plan, ca, sp.y, plan->n_samples, 0, N3, sp.We, sp.Mb, A));
      DIS_TRY(dis_coil_ifft1_combine(ctx, plan, ca, A, U, scale));
    }
    int nm = 0;
    if (motion)
      for (int s : segs)
        if (s < plan->n_mot) ++nm;
    DIS_TRY(sum_back(ctx, plan, U, sp.T, sp.T_n, segs, nm, &w, out, &first));
  }
  return DISORDER_OK;
}

// ---------------------------------------------------------------- per-state residuals
int dis_state_residual(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* y, const float2* Sf, int C,
                       const float2* x, const float* T, int n3_lo, int n3_hi, float2* r) {
  const long long V = plan->V;
  const int S = plan->n_mot;
  const int N3 = plan->N[2];
  const int N3c = n3_hi - n3_lo;
  DIS_CUDA_TRY(cudaMemsetAsync(r, 0, sizeof(float2) * plan->n_samples * N3 * C, ctx->stream));
  if (S == 0) return DISORDER_OK;
  const size_t per = (size_t)V * sizeof(float2) + coil_slot_bytes(plan, C, N3c) + dis_table_bytes(plan, 1, false);
  const int ch = (int)std::max<size_t>(1, std::min<size_t>(S, dis_budget_bytes() / per));
  for (int c0 = 0; c0 < S; c0 += ch) {
    const int n = std::min(ch, S - c0);
    std::vector<int> st(n);
    for (int j = 0; j < n; ++j) st[j] = c0 + j;
    Workspace w;
    DIS_TRY(dis_workspace(ctx, (size_t)n * per + (1 << 20), &w));
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, st, &d_seg));
    float2* z = w.take<float2>((size_t)n * V);
    float2* A = w.take<float2>((size_t)n * C * plan->N[0] * plan->N[1] * N3c);
    if (!z || !A) return dis_set_error(ctx, DISORDER_OOM, "state residual: workspace too small");
    std::vector<SlotParams> prm;
    dis_slot_params(T, S, st.data(), n, 1, &prm);
    Tables tb;
    DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w, &tb));
    DIS_TRY(dis_forward_transform(ctx, plan, x, 0, z, tb, 1, nullptr));
    DIS_TRY(dis_encode_volumes(ctx, plan, z, d_seg, st, Sf, C, n3_lo, N3c, A, r, plan->n_samples, n3_lo, N3, y));
  }
  return DISORDER_OK;
}

int dis_backproject_states(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* r, const float2* Sf,
                           int C, const float* T, float2* out) {
  const long long V = plan->V;
  const int S = plan->n_mot;
  const int N3 = plan->N[2];
  if (S == 0) return DISORDER_OK;
  std::vector<int> all(S);
  for (int j = 0; j < S; ++j) all[j] = j;
  const CoilPlan cp = coil_plan(plan, C, N3, all);
  const size_t coil = cp.sum ? cp.gather : cp.per_slot;
  const int ch = cp.sum ? chunk_for(plan, coil, 0, S) : dis_chunk_slots(plan, C, N3, 0, S);
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, (size_t)ch * coil + dis_table_bytes(plan, ch, false) + 4096 * 4, &ws));
  const float scale = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
  for (int c0 = 0; c0 < S; c0 += ch) {
    const int n = std::min(ch, S - c0);
    Workspace w = ws;
    std::vector<int> st(n);
    for (int j = 0; j < n; ++j) st[j] = c0 + j;
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, st, &d_seg));
    float2* U = out + (long long)c0 * V;
    CoilArgs ca = coil_args(plan, Sf, C, 0, N3, V, n, d_seg);
    if (cp.sum) {
      float2* Q = w.take<float2>((size_t)n * cp.gather / sizeof(float2));
      if (!Q) return dis_set_error(ctx, DISORDER_OOM, "back-projection: workspace too small");
      DIS_TRY(dis_coil_sum_adj(ctx, plan, ca, r, plan->n_samples, 0, N3, nullptr, nullptr, U, scale, Q, cp.ldp));
    } else {
      float2* A = w.take<float2>((size_t)n * C * V);
      if (!A) return dis_set_error(ctx, DISORDER_OOM, "back-projection: workspace too small");
      DIS_TRY(dis_coil_scatter_ifft2(ctx, plan, ca, r, plan->n_samples, 0, N3, nullptr, nullptr, A));
      DIS_TRY(dis_coil_ifft1_combine(ctx, plan, ca, A, U, scale));
    }
    if (dis_any_motion(T, S)) {
      std::vector<SlotParams> prm;
      dis_slot_params(T, S, st.data(), n, 0, &prm);
      Tables tb;
      DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w, &tb));
      DIS_TRY(dis_inverse_transform(ctx, plan, U, tb, 1, nullptr, 0.f));
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
  bool first = true;
  if (dis_plane_usable(plan, sp.C, sp.segs)) {
    if (sp.ys) return dis_set_error(ctx, DISORDER_BAD_ARG, "encodedecode: sample output needs the three-pass path");
    const int ch = plane_chunk(plan, nsg, V * sizeof(float2));
    Workspace ws;
    DIS_TRY(dis_workspace(ctx, (size_t)ch * V * sizeof(float2) + 2 * dis_table_bytes(plan, ch, false) + (1 << 20),
                          &ws));
    for (int c0 = 0; c0 < nsg; c0 += ch) {
      const int n = std::min(ch, nsg - c0);
      Workspace w = ws;
      std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
      int* d_seg = nullptr;
      DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
      float2* U = w.take<float2>((size_t)n * V);
      if (!U) return dis_set_error(ctx, DISORDER_OOM, "encodedecode: workspace too small");
      int nm = 0;
      if (motion) {
        std::vector<int> mot;
        for (int s : segs)
          if (s < plan->n_mot) mot.push_back(s);
        nm = (int)mot.size();
        if (nm) {
          std::vector<SlotParams> prm;
          dis_slot_params(sp.T, sp.T_n, mot.data(), nm, 1, &prm);
          Tables tb;
          DIS_TRY(dis_build_tables(ctx, plan, prm, false, &w, &tb));
          DIS_TRY(dis_forward_transform(ctx, plan, sp.x, 0, U, tb, 1, nullptr));
        }
        if (n > nm) DIS_TRY(dis_broadcast(ctx, sp.x, V, n - nm, U + (long long)nm * V));
        // the plane kernel reads each plane of U fully before writing it back
        DIS_TRY(plane_run(ctx, plan, pl::ENCDEC, U, V, U, V, sp.Sf, sp.C, 0, N3, d_seg, n, max_samples(plan, segs),
                          nullptr, nullptr, plan->n_samples, 0, N3, sp.We, nullptr));
      } else {
        DIS_TRY(plane_run(ctx, plan, pl::ENCDEC, sp.x, 0, U, V, sp.Sf, sp.C, 0, N3, d_seg, n, max_samples(plan, segs),
                          nullptr, nullptr, plan->n_samples, 0, N3, sp.We, nullptr));
      }
      DIS_TRY(sum_back(ctx, plan, U, sp.T, sp.T_n, segs, nm, &w, out, &first));
    }
    return DISORDER_OK;
  }
  const CoilPlan cp = coil_plan(plan, sp.C, N3, sp.segs);
  const int ch = chunk_for(plan, cp.per_slot, V * sizeof(float2), nsg);
  // the sample-sum stage goes through the samples E x: the caller's ys, or a
  // buffer of all samples (each chunk writes and reads its own segments' rows)
  const long long ny = plan->n_samples * N3 * (long long)sp.C;
  const size_t ybuf = (cp.sum && !sp.ys) ? ((size_t)ny * sizeof(float2) + 256) : 0;
  const size_t need = (size_t)ch * (cp.per_slot + V * sizeof(float2)) + 2 * dis_table_bytes(plan, ch, false) +
                      ybuf + 4096 * 4;
  Workspace ws;
  DIS_TRY(dis_workspace(ctx, need, &ws));
  float2* ysb = sp.ys;
  if (cp.sum && !ysb) {
    ysb = ws.take<float2>((size_t)ny);
    if (!ysb) return dis_set_error(ctx, DISORDER_OOM, "encodedecode: workspace too small");
  }
  for (int c0 = 0; c0 < nsg; c0 += ch) {
    const int n = std::min(ch, nsg - c0);
    Workspace w = ws;
    std::vector<int> segs(sp.segs.begin() + c0, sp.segs.begin() + c0 + n);
    int* d_seg = nullptr;
    DIS_TRY(dis_upload_ints(ctx, &w, segs, &d_seg));
    float2* A = w.take<float2>((size_t)n * cp.per_slot / sizeof(float2));
    if (!A) return dis_set_error(ctx, DISORDER_OOM, "encodedecode: workspace too small");
    const float2* z;
    long long Vz;
    float2* Z = nullptr;
    int nm;
    DIS_TRY(states_of(ctx, plan, sp.x, sp.T, sp.T_n, motion, segs, &w, &z, &Vz, &Z, &nm));
    float2* U = Z;
    if (!U) {
      U = w.take<float2>((size_t)n * V);
      if (!U) return dis_set_error(ctx, DISORDER_OOM, "encodedecode: workspace too small");
    }
    CoilArgs ca = coil_args(plan, sp.Sf, sp.C, 0, N3, Vz, n, d_seg);
    if (cp.sum) {
      // E x into the samples, then E^H W of them (encodedecode.m:125,133 apply EH.We)
      const float s1 = (float)(1.0 / std::sqrt((double)plan->N[0] * plan->N[1]));
      DIS_TRY(dis_coil_sum_fwd(ctx, plan, ca, z, A, cp.ldp, ysb, plan->n_samples, 0, N3, nullptr, s1));
      ca.Vz = V;
      // (the partial sums are reduced by now: their buffer takes the gathered samples)
      DIS_TRY(dis_coil_sum_adj(ctx, plan, ca, ysb, plan->n_samples, 0, N3, sp.We, nullptr, U, s1, A, cp.ldp));
    } else {
      DIS_TRY(dis_coil_expand_fft1(ctx, plan, ca, z, A));
      DIS_TRY(dis_coil_fft2_weight(ctx, plan, ca, A, sp.wmap, sp.ys, plan->n_samples, 0, N3));
      ca.Vz = V;
      const float scale = (float)(1.0 / ((double)plan->N[0] * plan->N[1]));
      DIS_TRY(dis_coil_ifft1_combine(ctx, plan, ca, A, U, scale));
    }
    DIS_TRY(sum_back(ctx, plan, U, sp.T, sp.T_n, segs, nm, &w, out, &first));
  }
  return DISORDER_OK;
}
