// Encoder driver specifications (internal).
#pragma once
#include <vector>

#include "internal.h"

struct EncodeSpec {
  const float2* x = nullptr;   // one volume
  const float2* Sf = nullptr;  // full-readout coil maps
  int C = 0;
  const float* T = nullptr;    // host, T_n x 6 parameter-major (NULL: no motion)
  int T_n = 0;
  std::vector<int> segs;       // segments to encode, motion segments first
  int n3_lo = 0, N3c = 0;      // readout range processed
  long long y_ld = 0;          // leading dim of y (total samples)
  int y_n3off = 0, y_N3 = 0;   // readout offset/extent of y's layout
};

struct DecodeSpec {
  const float2* y = nullptr;
  const float2* Sf = nullptr;
  int C = 0;
  const float* T = nullptr;
  int T_n = 0;
  std::vector<int> segs;
  const float* We = nullptr;
  const float* Mb = nullptr;
};

struct EncodeDecodeSpec {
  const float2* x = nullptr;
  const float2* Sf = nullptr;
  int C = 0;
  const float* T = nullptr;
  int T_n = 0;
  std::vector<int> segs;
  const float* wmap = nullptr;  // [seg][N1][N2] (kz fastest) sample weights of each grid point (three-pass path)
  const float* We = nullptr;    // per-sample weights (plane path), NULL for 1
  // when set (three-pass path only), the samples of the forward half, E x in
  // encode's layout (y_ld = n_samples, all readout rows), are written here
  float2* ys = nullptr;
};

size_t dis_budget_bytes();
bool dis_any_motion(const float* T, int n);
size_t dis_table_bytes(const disorder_plan_s* plan, int ns, bool grad);
int dis_chunk_slots(const disorder_plan_s* plan, int C, int N3c, size_t extra_per_slot, int n_total);
int dis_upload_ints(disorder_ctx_s* ctx, Workspace* ws, const std::vector<int>& v, int** out);
int dis_encode_segments(disorder_ctx_s* ctx, const disorder_plan_s* plan, const EncodeSpec& sp, float2* y,
                        const float2* y_meas);
int dis_encode_volumes(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* vols, const int* d_segs,
                       const std::vector<int>& segs, const float2* Sf, int C, int n3_lo, int N3c, float2* A, float2* y, long long y_ld,
                       int y_n3off, int y_N3, const float2* y_meas);
int dis_decode_segments(disorder_ctx_s* ctx, const disorder_plan_s* plan, const DecodeSpec& sp, float2* out);
// r = encode(T_s x) - y for every motion state over readout rows [n3_lo, n3_hi),
// the other rows zero (r: samples x N3 x C, encode's layout)
int dis_state_residual(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* y, const float2* Sf, int C,
                       const float2* x, const float* T, int n3_lo, int n3_hi, float2* r);
// out[s] = T_s^H sum_c S_c^H F^H r_s for every motion state s (not summed)
int dis_backproject_states(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* r, const float2* Sf,
                           int C, const float* T, float2* out);
int dis_encodedecode_segments(disorder_ctx_s* ctx, const disorder_plan_s* plan, const EncodeDecodeSpec& sp,
                              float2* out);
int dis_gradient(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* x, long long x_s,
                 const Tables& tb, float2* z, float2* yB, float2* w1, float2* w2, float2* G);
bool dis_plane_usable(const disorder_plan_s* plan, int C, const std::vector<int>& segs);
// the sample-sum coil stage (sumcoil.cu): no per-coil intermediate volumes
bool dis_sum_coil_usable(const disorder_plan_s* plan);
size_t dis_sum_part_bytes(const disorder_plan_s* plan, int C, int N3c, int ldp);
int dis_coil_sum_fwd(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* z,
                     float2* part, int ldp, float2* y, long long y_ld, int y_n3off, int y_N3, const float2* y_meas,
                     float scale);
size_t dis_sum_gather_bytes(int C, int N3c, int ldq);
int dis_coil_sum_adj(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* y,
                     long long y_ld, int y_n3off, int y_N3, const float* We, const float* Mb, float2* u, float scale,
                     float2* yq, int ldq);
int dis_sum_slots(disorder_ctx_s* ctx, const float2* u, long long V, int n_slots, float2* out, float beta);
int dis_broadcast(disorder_ctx_s* ctx, const float2* x, long long V, int n_slots, float2* out);
