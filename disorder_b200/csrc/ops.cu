// Host-side orchestration of the line passes: the sinc rigid transform
// (forward, inverse, gradient) and the encoding operators.
#include <algorithm>
#include <cmath>

#include "internal.h"

namespace {

const int TR0[3] = {0, 2, 1};  // tr(1,:) (Methods/sincRigidTransform.m:33-34), 0-based
const int TR1[3] = {1, 0, 2};  // tr(2,:)

LinePassArgs base_args(const disorder_plan_s* plan, int axis, int n_slots) {
  LinePassArgs a;
  for (int i = 0; i < 3; ++i) a.N[i] = plan->N[i];
  a.axis = axis;
  a.L = 0;
  a.pitch = 0;
  a.n_slots = n_slots;
  a.accumulate = 0;
  a.beta = 0.f;
  a.in0 = a.in1 = nullptr;
  a.out0 = a.out1 = nullptr;
  a.in0_s = a.in1_s = a.out0_s = a.out1_s = 0;
  a.c00 = a.c01 = a.c10 = a.c11 = P_ZERO;
  a.Sd = TabRef();
  a.sd_w = 0;
  a.kG = plan->d_kG[axis];
  a.tw = plan->d_tw[axis];
  a.plan = plan->fft[axis];
  return a;
}

TabRef tab(const float2* p, long long s, int b) {
  TabRef t;
  t.p = p;
  t.sstride = s;
  t.b = b;
  return t;
}

// one shear pass of rotation m: which = 0 -> e2 along a1 (row from a2),
// which = 1 -> e3 along a2 (row from a1)
LinePassArgs shear_args(const disorder_plan_s* plan, const Tables& tb, int m, int which, int n_slots) {
  const int a1 = TR0[m], a2 = TR1[m];
  LinePassArgs a = base_args(plan, which == 0 ? a1 : a2, n_slots);
  if (which == 0) {
    a.A = tab(tb.e2[m], tb.e2s[m], a2);
    a.B = tab(tb.g2[m], tb.e2s[m], a2);
    a.Sd = tab(tb.sd2[m], tb.sd2s[m], a2);
    a.sd_w = tb.sdw[a1];
  } else {
    a.A = tab(tb.e3[m], tb.e3s[m], a1);
    a.B = tab(tb.g3[m], tb.e3s[m], a1);
    a.Sd = tab(tb.sd3[m], tb.sd3s[m], a1);
    a.sd_w = tb.sdw[a2];
  }
  a.c00 = P_A;
  return a;
}

// The coefficient setters below keep the table form (A, T) and the seed
// form (Sd) of a pass in step.
// translation-only pass along ax: (1/N) et{1}{ax}
void set_translation(LinePassArgs& a, const Tables& tb, int ax) {
  a.c00 = P_ONE;
  a.T = tab(tb.e1[ax], tb.e1s[ax], -1);
  a.Sd = tab(tb.sd1[ax], tb.sd1s[ax], -1);
  a.sd_w = tb.sdw[ax];
}

// et{1}{2} fused into the last e2 pass of rotation 3 (single-input form)
void fuse_t1(LinePassArgs& a, const Tables& tb) {
  a.T = tab(tb.e1[1], tb.e1s[1], -1);
  a.Sd = tab(tb.sd2t, tb.sd2ts, TR1[2]);
}

void io(LinePassArgs& a, const float2* in, long long in_s, float2* out, long long out_s) {
  a.in0 = in;
  a.in0_s = in_s;
  a.out0 = out;
  a.out0_s = out_s;
}

__global__ void sum_slots_kernel(const float2* __restrict__ u, long long V, int n_slots, float2* __restrict__ out,
                                 float beta) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < V; i += (long long)gridDim.x * blockDim.x) {
    float2 acc = beta != 0.f ? cscale(out[i], beta) : make_float2(0.f, 0.f);
    for (int j = 0; j < n_slots; ++j) acc = cadd(acc, u[j * V + i]);
    out[i] = acc;
  }
}

__global__ void broadcast_kernel(const float2* __restrict__ x, long long V, int n_slots, float2* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < V; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = x[i];
    for (int j = 0; j < n_slots; ++j) out[j * V + i] = v;
  }
}

int sum_slots(disorder_ctx_s* ctx, const float2* u, long long V, int n_slots, float2* out, float beta) {
  const int blocks = (int)std::min<long long>((V + 255) / 256, 8LL * ctx->sm_count);
  sum_slots_kernel<<<blocks, 256, 0, ctx->stream>>>(u, V, n_slots, out, beta);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int broadcast(disorder_ctx_s* ctx, const float2* x, long long V, int n_slots, float2* out) {
  const int blocks = (int)std::min<long long>((V + 255) / 256, 8LL * ctx->sm_count);
  broadcast_kernel<<<blocks, 256, 0, ctx->stream>>>(x, V, n_slots, out);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

int flips(disorder_ctx_s* ctx, const disorder_plan_s* plan, const Tables& tb, int m, float2* vols) {
  if (!tb.any_flip[m]) return DISORDER_OK;
  const int n = (int)tb.flip_slots[m].size();
  // flipping(x, et{4}{m}) acts on the two axes of rotation m (flipping.m:11-22)
  DIS_TRY(dis_flip_pass(ctx, plan, vols, plan->V, tb.d_flip_slots[m], n, TR0[m], plan->cent[TR0[m]]));
  DIS_TRY(dis_flip_pass(ctx, plan, vols, plan->V, tb.d_flip_slots[m], n, TR1[m], plan->cent[TR1[m]]));
  return DISORDER_OK;
}

// the rotations m0..2 and the translation applied in place to w (per-slot
// volumes); rotation m0's flip is applied first. The last pass writes `out`.
int rotations_and_translation(disorder_ctx_s* ctx, const disorder_plan_s* plan, const Tables& tb, int m0,
                              float2* w, float2* out) {
  const long long V = plan->V;
  const int ns = tb.n_slots;
  for (int m = m0; m < 3; ++m) {
    DIS_TRY(flips(ctx, plan, tb, m, w));
    LinePassArgs a = shear_args(plan, tb, m, 0, ns);
    io(a, w, V, w, V);
    DIS_TRY(dis_line_pass(ctx, a));
    a = shear_args(plan, tb, m, 1, ns);
    io(a, w, V, w, V);
    DIS_TRY(dis_line_pass(ctx, a));
    a = shear_args(plan, tb, m, 0, ns);
    io(a, w, V, w, V);
    if (m == 2) fuse_t1(a, tb);
    DIS_TRY(dis_line_pass(ctx, a));
  }
  LinePassArgs a = base_args(plan, 0, ns);
  set_translation(a, tb, 0);
  io(a, w, V, w, V);
  DIS_TRY(dis_line_pass(ctx, a));
  a = base_args(plan, 2, ns);
  set_translation(a, tb, 2);
  io(a, w, V, out, V);
  DIS_TRY(dis_line_pass(ctx, a));
  return DISORDER_OK;
}

}  // namespace

// Forward transform (sincRigidTransform.m:38-75) of x (per-slot stride x_s,
// 0 = one shared volume) into z (n_slots volumes). When yB is given it must
// hold 2 volumes per slot: yB[0..ns) receives the state before rotation 2
// (after its flip) and yB[ns..2ns) the state before rotation 3, the image-space
// forms of the reference's xB{2} and xB{3}; xB{1} is the input itself.
int dis_forward_transform(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* x, long long x_s,
                          float2* z, const Tables& tb, int useFull, float2* yB) {
  const long long V = plan->V;
  const int ns = tb.n_slots;
  if (ns == 0) return DISORDER_OK;
  const float2* cur = x;
  long long cur_s = x_s;
  if (useFull == 0) {
    // translations only: DFT along every axis, et{1}, inverse DFT (:59-64)
    for (int ax = 0; ax < 3; ++ax) {
      LinePassArgs a = base_args(plan, ax, ns);
      set_translation(a, tb, ax);
      io(a, cur, cur_s, z, V);
      DIS_TRY(dis_line_pass(ctx, a));
      cur = z;
      cur_s = V;
    }
    return DISORDER_OK;
  }
  for (int m = 0; m < 3; ++m) {
    if (tb.any_flip[m]) {
      if (cur != z) {
        if (cur_s == 0) {
          DIS_TRY(broadcast(ctx, cur, V, ns, z));
        } else {
          DIS_CUDA_TRY(cudaMemcpyAsync(z, cur, sizeof(float2) * V * ns, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        cur = z;
        cur_s = V;
      }
      DIS_TRY(flips(ctx, plan, tb, m, z));
    }
    if (yB && m > 0) {
      // record the state entering rotation m (image space)
      float2* dst = yB + (long long)(m - 1) * ns * V;
      if (cur != dst) DIS_CUDA_TRY(cudaMemcpyAsync(dst, cur, sizeof(float2) * V * ns, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    LinePassArgs a = shear_args(plan, tb, m, 0, ns);
    io(a, cur, cur_s, z, V);
    DIS_TRY(dis_line_pass(ctx, a));
    a = shear_args(plan, tb, m, 1, ns);
    io(a, z, V, z, V);
    DIS_TRY(dis_line_pass(ctx, a));
    a = shear_args(plan, tb, m, 0, ns);
    io(a, z, V, z, V);
    if (m == 2 && useFull != -1) fuse_t1(a, tb);  // et{1}{2} fused (:57-72)
    DIS_TRY(dis_line_pass(ctx, a));
    cur = z;
    cur_s = V;
  }
  if (useFull != -1) {
    LinePassArgs a = base_args(plan, 0, ns);
    set_translation(a, tb, 0);
    io(a, z, V, z, V);
    DIS_TRY(dis_line_pass(ctx, a));
    a = base_args(plan, 2, ns);
    set_translation(a, tb, 2);
    io(a, z, V, z, V);
    DIS_TRY(dis_line_pass(ctx, a));
  }
  return DISORDER_OK;
}

// Inverse transform (sincRigidTransform.m:76-113) applied in place to the
// n_slots volumes u. With out != nullptr the states are summed into out as
// out = beta*out + sum_slots (fused into the last pass when no flip follows).
int dis_inverse_transform(disorder_ctx_s* ctx, const disorder_plan_s* plan, float2* u, const Tables& tb,
                          int useFull, float2* out, float beta) {
  const long long V = plan->V;
  const int ns = tb.n_slots;
  if (ns == 0) {
    if (out && beta == 0.f) DIS_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float2) * V, ctx->stream));
    return DISORDER_OK;
  }
  if (useFull == 0) {
    for (int ax = 0; ax < 3; ++ax) {
      LinePassArgs a = base_args(plan, ax, ns);
      set_translation(a, tb, ax);
      io(a, u, V, u, V);
      if (ax == 2 && out) {
        a.accumulate = 1;
        a.beta = beta;
        a.out0 = out;
      }
      DIS_TRY(dis_line_pass(ctx, a));
    }
    return DISORDER_OK;
  }
  if (useFull != -1) {
    for (int ax : {2, 0}) {
      LinePassArgs a = base_args(plan, ax, ns);
      set_translation(a, tb, ax);
      io(a, u, V, u, V);
      DIS_TRY(dis_line_pass(ctx, a));
    }
  }
  bool summed = false;
  for (int m = 2; m >= 0; --m) {
    LinePassArgs a = shear_args(plan, tb, m, 0, ns);
    io(a, u, V, u, V);
    if (m == 2 && useFull != -1) fuse_t1(a, tb);
    DIS_TRY(dis_line_pass(ctx, a));
    a = shear_args(plan, tb, m, 1, ns);
    io(a, u, V, u, V);
    DIS_TRY(dis_line_pass(ctx, a));
    a = shear_args(plan, tb, m, 0, ns);
    io(a, u, V, u, V);
    if (m == 0 && out && !tb.any_flip[0]) {
      a.accumulate = 1;
      a.beta = beta;
      a.out0 = out;
      summed = true;
    }
    DIS_TRY(dis_line_pass(ctx, a));
    DIS_TRY(flips(ctx, plan, tb, m, u));
  }
  if (out && !summed) DIS_TRY(sum_slots(ctx, u, V, ns, out, beta));
  return DISORDER_OK;
}

// sincRigidTransformGradient (Methods/sincRigidTransformGradient.m:19-149).
// x: one volume (shared) or per-slot volumes (x_s); G: 6 blocks of ns volumes.
// Work buffers: z (ns vols), yB (2*ns vols), w1, w2 (ns vols each).
int dis_gradient(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* x, long long x_s,
                 const Tables& tb, float2* z, float2* yB, float2* w1, float2* w2, float2* G) {
  const long long V = plan->V;
  const int ns = tb.n_slots;
  if (ns == 0) return DISORDER_OK;
  const long long Gs = (long long)ns * V;
  // the transform and its intermediates
  const float2* in0 = x;
  long long in0_s = x_s;
  if (tb.any_flip[0]) {
    // xB{1} is the flipped input; materialise it per slot in w2 first
    if (x_s == 0) {
      DIS_TRY(broadcast(ctx, x, V, ns, w2));
    } else {
      DIS_CUDA_TRY(cudaMemcpyAsync(w2, x, sizeof(float2) * V * ns, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    DIS_TRY(flips(ctx, plan, tb, 0, w2));
    in0 = w2;
    in0_s = V;
  }
  // forward with the flip of rotation 0 already applied to in0
  {
    Tables tb2 = tb;
    tb2.any_flip[0] = false;
    DIS_TRY(dis_forward_transform(ctx, plan, in0, in0_s, z, tb2, 1, yB));
  }
  // translations: G{m} = IFFT_m(-i k_m FFT_m(z)) (:29-36)
  for (int ax = 0; ax < 3; ++ax) {
    LinePassArgs a = base_args(plan, ax, ns);
    a.c00 = P_DK;
    io(a, z, V, G + ax * Gs, V);
    DIS_TRY(dis_line_pass(ctx, a));
  }
  // rotation m: start from the state entering rotation m
  for (int m = 0; m < 3; ++m) {
    const float2* src = (m == 0) ? in0 : yB + (long long)(m - 1) * ns * V;
    const long long src_s = (m == 0) ? in0_s : V;
    const int a1 = TR0[m], a2 = TR1[m];
    // P1: X = F_a1(src); w1 = IF(e2 X), w2 = IF(etg2 X)
    LinePassArgs a = base_args(plan, a1, ns);
    a.A = tab(tb.e2[m], tb.e2s[m], a2);
    a.B = tab(tb.g2[m], tb.e2s[m], a2);
    a.c00 = P_A;
    a.c10 = P_B;
    a.in0 = src;
    a.in0_s = src_s;
    a.out0 = w1;
    a.out0_s = V;
    a.out1 = (m == 0 && tb.any_flip[0]) ? z : w2;  // w2 may hold the flipped input
    a.out1_s = V;
    float2* w2m = a.out1;
    DIS_TRY(dis_line_pass(ctx, a));
    // P2: along a2: w2 = IF(etg3 F w1 + e3 F w2), w1 = IF(e3 F w1)
    a = base_args(plan, a2, ns);
    a.A = tab(tb.e3[m], tb.e3s[m], a1);
    a.B = tab(tb.g3[m], tb.e3s[m], a1);
    a.c00 = P_A;
    a.c10 = P_B;
    a.c11 = P_A;
    a.in0 = w1;
    a.in0_s = V;
    a.in1 = w2m;
    a.in1_s = V;
    a.out0 = w1;
    a.out0_s = V;
    a.out1 = w2m;
    a.out1_s = V;
    DIS_TRY(dis_line_pass(ctx, a));
    // P3: along a1: w1 = IF(etg2 F w1 + e2 F w2) (x e1{2} for the last rotation)
    a = base_args(plan, a1, ns);
    a.A = tab(tb.e2[m], tb.e2s[m], a2);
    a.B = tab(tb.g2[m], tb.e2s[m], a2);
    a.c00 = P_B;
    a.c01 = P_A;
    a.in0 = w1;
    a.in0_s = V;
    a.in1 = w2m;
    a.in1_s = V;
    a.out0 = w1;
    a.out0_s = V;
    if (m == 2) a.T = tab(tb.e1[1], tb.e1s[1], -1);
    DIS_TRY(dis_line_pass(ctx, a));
    float2* g = G + (3 + m) * Gs;
    if (m < 2) {
      DIS_TRY(rotations_and_translation(ctx, plan, tb, m + 1, w1, g));
    } else {
      LinePassArgs t = base_args(plan, 0, ns);
      set_translation(t, tb, 0);
      io(t, w1, V, w1, V);
      DIS_TRY(dis_line_pass(ctx, t));
      t = base_args(plan, 2, ns);
      set_translation(t, tb, 2);
      io(t, w1, V, g, V);
      DIS_TRY(dis_line_pass(ctx, t));
    }
  }
  return DISORDER_OK;
}

// -------------------------------------------------------------- helpers used by the encoders
int dis_sum_slots(disorder_ctx_s* ctx, const float2* u, long long V, int n_slots, float2* out, float beta) {
  return sum_slots(ctx, u, V, n_slots, out, beta);
}
int dis_broadcast(disorder_ctx_s* ctx, const float2* x, long long V, int n_slots, float2* out) {
  return broadcast(ctx, x, V, n_slots, out);
}
