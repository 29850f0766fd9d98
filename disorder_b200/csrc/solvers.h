// Solver specifications (internal).
#pragma once
#include "internal.h"

struct CGSpec {
  const float2* y = nullptr;
  const float2* Sf = nullptr;
  int C = 0;
  const float* T = nullptr;  // host n_mot x 6 or NULL
  const float* We = nullptr;
  const float* Mb = nullptr;
  const float* Mbe = nullptr;
  const float* P_Se = nullptr;
  const float* C_Ma = nullptr;
  const float* R_Ti = nullptr;
  float2* r_out = nullptr;  // device, optional: the final sample residual E x - y (encode's layout)
  // shearlet term of regularize.m:27-46 (CSsolver.m:76): sh_scale = la p / 2
  const disorder_shearlet_s* sh = nullptr;
  const float* sh_We = nullptr;
  float sh_scale = 0.f;
};

struct LMSpec {
  const float2* y = nullptr;
  const float2* Sf = nullptr;
  int C = 0;
  const float2* x = nullptr;
  float winit = 1e-3f;
  float tL[2] = {0.f, 0.f};
  int n3_lo = 0, n3_hi = 0;
};

// out = beta out + scale IDFT3(sum_w S_w .* DFT3(We_w .* IDFT3(conj(S_w) .* DFT3(x)))) (shearlet.cu)
int dis_shearlet_regularize(disorder_ctx_s* ctx, const disorder_shearlet_s* sh, const float2* x, const float* We,
                            float scale, float beta, float2* out);

disorder_ctx_s* dis_shearlet_ctx(const disorder_shearlet_s* sh);
void dis_shearlet_size(const disorder_shearlet_s* sh, int* N);

int dis_cg_solve(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CGSpec& s, float2* x, int x_init, int nIt,
                 int tolType, double tol, double* En, int* n_en, int* nn);
int dis_lm_step(disorder_ctx_s* ctx, const disorder_plan_s* plan, const LMSpec& s, float* T, float* w, uint8_t* cT,
                double* En, double* EnPrev);
int dis_energy(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* y, const float2* x, const float2* Sf,
               int C, const float* T, const float* rowW, const float* R_Ti, float2* rbuf, double* En, int n3_lo = 0,
               int n3_cnt = -1);
// fidelity of a residual r = E x - y (encode's layout): sum of rowW[n3] |r|^2
// over rows [n3_lo, n3_lo + n3_cnt) (n3_cnt < 0 or no rowW: all rows, weight 1)
int dis_fidelity(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* rbuf, int C, const float* rowW,
                 double* En, int n3_lo = 0, int n3_cnt = -1);
int dis_ti_energy(disorder_ctx_s* ctx, const float2* x, const float* ti, long long n, double* out);
int dis_weighted_norm(disorder_ctx_s* ctx, const float2* b, const float* w, long long n, double* out);
