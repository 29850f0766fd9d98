// Shared definitions of the shearlet passes (shearlet.cu) and the
// register-FFT pass kernel, instantiated per line length and pass kind in
// shearlet_fa.cu / shearlet_fb.cu.
#pragma once
#include <vector>

#include "fastfft.cuh"
#include "fft.cuh"
#include "internal.h"
#include "tiles.cuh"

struct disorder_shearlet_s {
  disorder_ctx_s* ctx = nullptr;
  int N[3] = {0, 0, 0};
  int n_planes = 0;
  int n_filters = 0;
  float2* planes = nullptr;   // pair blocks, each n_planes planes of Na x Nb (column-major)
  long long pair_off[3] = {0, 0, 0};
  long long plane_size[3] = {0, 0, 0};
  std::vector<int> table;     // n_filters x 4: pair A, plane A, pair B, plane B
  float2* tw[3] = {nullptr, nullptr, nullptr};  // W_N^m of each axis length (device)
};

namespace shl {

constexpr int kThr = 256;
// the dimension pairs of the 2-D planes (0-based), first dimension fastest
constexpr int kPair[3][2] = {{0, 1}, {0, 2}, {2, 1}};

enum { PRE_NONE = 0, PRE_CONJ_FILTER = 1, PRE_COIL = 2 };
enum {
  POST_STORE = 0,       // out = v
  POST_TIMES_WE = 1,    // out = We .* v
  POST_COEF = 2,        // we_out = (|v| + eps)^pw
  POST_ACC_FILTER = 3,  // acc += S_w .* v
  POST_TRACE_WE = 4,    // sum += We |v|^2
  POST_TRACE_GRID = 5,  // sum += scale W(k1, k2) |v|^2
  POST_AXPBY = 6        // out = beta out + scale v
};

struct ShFilt {
  const float2* A = nullptr;
  const float2* B = nullptr;
  int pa = 0, pb = 0;
};

struct ShArgs {
  int N[3];
  int axis = 0;
  int inv = 0;  // inverse DFT (1/n scaled)
  FFTPlan plan;
  int L = 16, P = 17;
  const float2* in = nullptr;
  const float* in_real = nullptr;  // real input instead of `in`
  float2* out = nullptr;
  int pre = PRE_NONE;
  const float2* pre_c = nullptr;
  int post = POST_STORE;
  // round trip inside the tile: inverse DFT, times mid_we (real, per voxel),
  // forward DFT, then the post step (the regularizer's last inverse and first
  // forward pass along the same axis in one pass)
  const float* mid_we = nullptr;
  const float* we = nullptr;
  float* we_out = nullptr;
  float eps = 0.f, pw = -1.f;
  float2* acc = nullptr;
  const float* wgrid = nullptr;
  float beta = 0.f, scale = 1.f;
  ShFilt f;
  double* sum = nullptr;
  const float2* twg = nullptr;  // device W_N^m of the axis length (register-FFT kernel), or null
};

DIS_D int pair_index(int q, int c0, int c1, int c2, const int* N) {
  return q == 0 ? c0 + N[0] * c1 : (q == 1 ? c0 + N[0] * c2 : c2 + N[2] * c1);
}

DIS_D float2 filter_at(const ShFilt& f, int c0, int c1, int c2, const int* N) {
  return cmul(f.A[pair_index(f.pa, c0, c1, c2, N)], f.B[pair_index(f.pb, c0, c1, c2, N)]);
}

// The pass kinds of the register-FFT kernel (a kernel per kind keeps each
// instantiation's registers to its own element-wise steps):
enum {
  K_FWD = 0,          // forward DFT, store
  K_FWD_ACC = 1,      // forward DFT, acc += S_w .* v
  K_INV_FILT = 2,     // conj(S_w) .* on load, inverse DFT, store
  K_INV = 3,          // inverse DFT, store
  K_INV_AXPBY = 4,    // inverse DFT, out = beta out + scale v
  K_INV_COEF = 5,     // inverse DFT, coefficient (|v| + eps)^pw
  K_INV_TRACE = 6,    // inverse DFT, sum += We |v|^2
  K_ROUND_TRIP = 7,   // inverse DFT, .* We, forward DFT, store
  K_COUNT = 8
};

// the kind of a pass, or -1 when the generic kernel must run it
inline int fast_kind(const ShArgs& a) {
  if (a.in_real || a.pre == PRE_COIL) return -1;
  if (a.mid_we) return (a.inv && a.pre == PRE_NONE && a.post == POST_STORE) ? K_ROUND_TRIP : -1;
  if (!a.inv) {
    if (a.pre != PRE_NONE) return -1;
    return a.post == POST_STORE ? K_FWD : (a.post == POST_ACC_FILTER ? K_FWD_ACC : -1);
  }
  if (a.pre == PRE_CONJ_FILTER) return a.post == POST_STORE ? K_INV_FILT : -1;
  switch (a.post) {
    case POST_STORE: return K_INV;
    case POST_AXPBY: return K_INV_AXPBY;
    case POST_COEF: return K_INV_COEF;
    case POST_TRACE_WE: return K_INV_TRACE;
    default: return -1;
  }
}

// Register-FFT form of a pass for lengths N = F1 * F2 with a fast
// factorisation (ff::Line, the four-step FFT of the transform's line passes):
// TL threads per line, LPB = 256 / TL lines per tile (adjacent along dim 1
// for the strided axes, so a row of the tile is contiguous), one tile per
// CTA. Forward passes read natural order into layout A (thread t < F2 holds
// x[t + F2 m]) and write the spectrum from layout B (thread k1 < F1 holds
// X[k1 + F1 k2]); inverse passes the other way round; the round trip reads
// and writes layout B.
template <int F1, int F2, int KIND>
__global__ void __launch_bounds__(kThr) sh_fast_kernel(ShArgs a) {
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, TL = LN::TL, LPB = kThr / TL;
  constexpr bool IN_B = KIND >= K_INV_FILT;                       // spectrum in
  constexpr bool OUT_B = KIND <= K_FWD_ACC || KIND == K_ROUND_TRIP;  // spectrum out
  extern __shared__ float2 sm[];
  __shared__ double red[kThr / 32];
  float2* twf = sm;                          // W_N^m, m < N
  float2* tws = twf + ((N + 1) & ~1);        // the line FFT's twiddles
  float2* exa = tws + ((LN::TWS + 1) & ~1);  // LPB exchange tiles
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  if (a.twg) {
    ff::load_tw<F1, F2>(tws, a.twg, tid, kThr);
  } else {
    for (int m = tid; m < N; m += kThr) {
      double sn, cs;
      sincospi(-2.0 * (double)m / (double)N, &sn, &cs);
      twf[m] = make_float2((float)cs, (float)sn);
    }
    __syncthreads();
    ff::load_tw<F1, F2>(tws, twf, tid, kThr);
  }
  __syncthreads();
  float2* ex = exa + li * LN::EXSZ;
  const int axis = a.axis;
  const long long st = axis == 0 ? 1LL : (axis == 1 ? (long long)a.N[0] : (long long)a.N[0] * a.N[1]);
  const int tile = blockIdx.x;
  long long base = 0;
  int c0 = 0, c1 = 0, c2 = 0;
  bool valid;
  if (axis == 0) {
    long long q = (long long)tile * LPB + li;
    valid = q < (long long)a.N[1] * a.N[2];
    if (!valid) q = 0;
    c1 = (int)(q % a.N[1]);
    c2 = (int)(q / a.N[1]);
    base = q * a.N[0];
  } else {
    const int nt0 = (a.N[0] + LPB - 1) / LPB;
    const int other = tile / nt0;
    c0 = (tile - other * nt0) * LPB + li;
    valid = c0 < a.N[0];
    if (!valid) c0 = 0;
    if (axis == 1) {
      c2 = other;
      base = c0 + (long long)c2 * a.N[0] * a.N[1];
    } else {
      c1 = other;
      base = c0 + (long long)c1 * a.N[0];
    }
  }
  // the filter S_w at position p of this line
  auto filt = [&](int p) {
    const int d0 = axis == 0 ? p : c0, d1 = axis == 1 ? p : c1, d2 = axis == 2 ? p : c2;
    return cmul(a.f.A[pair_index(a.f.pa, d0, d1, d2, a.N)], a.f.B[pair_index(a.f.pb, d0, d1, d2, a.N)]);
  };
  const float invn = 1.0f / (float)N;
  float2 A[F1], B[F2];
  if (IN_B) {
#pragma unroll
    for (int k2 = 0; k2 < F2; ++k2) {
      const int p = lt + F1 * k2;
      float2 v = make_float2(0.f, 0.f);
      if (valid && lt < F1) {
        v = a.in[base + p * st];
        if (KIND == K_INV_FILT) v = cmul(v, cconj(filt(p)));
      }
      B[k2] = v;
    }
    LN::inv(B, A, lt, ex, tws);
    if (KIND == K_ROUND_TRIP) {
#pragma unroll
      for (int m = 0; m < F1; ++m)
        A[m] = (valid && lt < F2) ? cscale(A[m], invn * a.mid_we[base + (lt + F2 * m) * st]) : make_float2(0.f, 0.f);
      LN::fwd(A, B, lt, ex, tws);
    } else {
#pragma unroll
      for (int m = 0; m < F1; ++m) A[m] = cscale(A[m], invn);
    }
  } else {
#pragma unroll
    for (int m = 0; m < F1; ++m) A[m] = (valid && lt < F2) ? a.in[base + (lt + F2 * m) * st] : make_float2(0.f, 0.f);
    LN::fwd(A, B, lt, ex, tws);
  }
  double part = 0.0;
  auto post = [&](int p, float2 v) {
    const long long g = base + p * st;
    if (KIND == K_FWD || KIND == K_INV || KIND == K_INV_FILT || KIND == K_ROUND_TRIP) {
      a.out[g] = v;
    } else if (KIND == K_FWD_ACC) {
      a.acc[g] = cadd(a.acc[g], cmul(filt(p), v));
    } else if (KIND == K_INV_AXPBY) {
      float2 o = cscale(v, a.scale);
      if (a.beta != 0.f) o = cadd(o, cscale(a.out[g], a.beta));
      a.out[g] = o;
    } else if (KIND == K_INV_COEF) {
      const float m = hypotf(v.x, v.y) + a.eps;
      a.we_out[g] = a.pw == -1.f ? 1.f / m : powf(m, a.pw);
    } else {
      part += (double)a.we[g] * ((double)v.x * v.x + (double)v.y * v.y);
    }
  };
  if (valid) {
    if (OUT_B) {
      if (lt < F1) {
#pragma unroll
        for (int k2 = 0; k2 < F2; ++k2) post(lt + F1 * k2, B[k2]);
      }
    } else if (lt < F2) {
#pragma unroll
      for (int m = 0; m < F1; ++m) post(lt + F2 * m, A[m]);
    }
  }
  if (KIND == K_INV_TRACE) {
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    if (tid == 0) {
      double t = 0;
      for (int w = 0; w < kThr / 32; ++w) t += red[w];
      atomicAdd(a.sum, t);
    }
  }
}

template <int F1, int F2, int KIND>
bool sh_fast_launch_kind(disorder_ctx_s* ctx, const ShArgs& a) {
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, LPB = kThr / LN::TL;
  const size_t smem = sizeof(float2) * (((N + 1) & ~1) + ((LN::TWS + 1) & ~1) + (size_t)LPB * LN::EXSZ);
  // set once per process (thread-safe static initialisation)
  static const cudaError_t attr =
      cudaFuncSetAttribute(sh_fast_kernel<F1, F2, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  (void)attr;
  const long long tiles = a.axis == 0 ? ((long long)a.N[1] * a.N[2] + LPB - 1) / LPB
                                      : (long long)((a.N[0] + LPB - 1) / LPB) * (a.axis == 1 ? a.N[2] : a.N[1]);
  if (tiles <= 0 || tiles >= (1LL << 31)) return false;
  sh_fast_kernel<F1, F2, KIND><<<(unsigned)tiles, kThr, smem, ctx->stream>>>(a);
  return true;
}

// the register-FFT pass of length F1*F2 for a.kind; false: not applicable
template <int F1, int F2>
bool sh_fast_launch(disorder_ctx_s* ctx, const ShArgs& a, int kind) {
  switch (kind) {
    case K_FWD: return sh_fast_launch_kind<F1, F2, K_FWD>(ctx, a);
    case K_FWD_ACC: return sh_fast_launch_kind<F1, F2, K_FWD_ACC>(ctx, a);
    case K_INV_FILT: return sh_fast_launch_kind<F1, F2, K_INV_FILT>(ctx, a);
    case K_INV: return sh_fast_launch_kind<F1, F2, K_INV>(ctx, a);
    case K_INV_AXPBY: return sh_fast_launch_kind<F1, F2, K_INV_AXPBY>(ctx, a);
    case K_INV_COEF: return sh_fast_launch_kind<F1, F2, K_INV_COEF>(ctx, a);
    case K_INV_TRACE: return sh_fast_launch_kind<F1, F2, K_INV_TRACE>(ctx, a);
    case K_ROUND_TRIP: return sh_fast_launch_kind<F1, F2, K_ROUND_TRIP>(ctx, a);
    default: return false;
  }
}

// instantiated in shearlet_fa.cu (256, 176, 128) and shearlet_fb.cu (88, 64, 44)
bool sh_fast_a(disorder_ctx_s* ctx, const ShArgs& a, int kind);
bool sh_fast_b(disorder_ctx_s* ctx, const ShArgs& a, int kind);

}  // namespace shl
