// Coil stage of the encoding operators without per-coil intermediate volumes.
//
// encode (Reconstruction/encode.m:90-136) evaluates, per motion state s, coil
// c and readout position n3, the unitary 2-D DFT of S_c .* z_s at the state's
// samples (ky_i, kz_i) only:
//   y_i = (N1 N2)^(-1/2) sum_b W2^{kz_i b} X[ky_i, b],  X = FFT_1(S_c .* z_s),
// and decode (decode.m:42-58,78-85) is its adjoint. The three-pass coil stage
// writes X for every coil (8 V C bytes per state) and reads it back three
// times. Here the dim-2 sum is split over tiles of LPB adjacent b (the lines
// of one CTA, along dim 1):
//   forward: a CTA loads its LPB lines of z_s once, and per coil multiplies by
//     S_c, FFTs along dim 1 in registers, puts X[b, ky] in shared memory and
//     adds sum_{b in tile} W2^{kz_i b} X[b, ky_i] for every sample i of the
//     state (threads walk the samples in ky order, so a warp reads a few
//     neighbouring rows of X); the tile's partial sums go to a buffer
//     part[slot][tile][c][n3][q] (q: the sample's place in ky order), and a
//     reduction adds the N2 / LPB tiles into y (times the DFT scale, minus the
//     measured samples when given);
//   adjoint: per coil the CTA rebuilds its LPB columns of X from the samples,
//     one thread per ky row and half of the lines (each row's samples are
//     contiguous in ky order, so no two threads write the same element),
//     X[b, ky] = sum_{i in row ky}
//     w_i y_i conj(W2^{kz_i b}), inverse-FFTs along dim 1 and accumulates
//     conj(S_c) .* (...) over the coils in registers; one store of u.
// Per state this moves 8 V (z) + 8 V (u) + the coil maps (shared by the
// states of a tile through L2) + the partial sums (N2 / LPB x the samples),
// against 40 V C for the three passes.
#include <cmath>

#include "encoding.h"
#include "fastpass.cuh"
#include "fastpass.h"
#include "internal.h"

namespace sc {

using fp::kThreads;

struct SumArgs {
  int N1, N2, N3c;
  long long Vz;          // slot stride of z / u
  const float2* Sf;      // coil maps, offset to the chunk's first readout row
  long long Sc;          // coil stride of Sf
  int C;
  int n_slots;
  const int* slot_seg;   // segment of each slot
  const int* rowptr;     // per-segment CSR over ky rows (global sample positions)
  const int* perm;       // sample index at each CSR position
  const int* kyq;        // its ky and kz
  const int* kzq;
  const float2* tw2;     // W_N2^m, m < N2
  float2* part;          // forward: [slot][tile][c][n3][q]; adjoint: the weighted samples [slot][c][n3][q]
  int ldp;               // q stride (most samples of a chunk segment)
  int ntile;             // N2 / LPB
};

// lane-wise a * b + c and a * b on (x, y) float pairs: one packed f32x2 op
DIS_D float2 pfma(float2 a, float2 b, float2 c) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pc, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "mov.b64 pc, {%6, %7};\n\tfma.rn.f32x2 pd, pa, pb, pc;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return r;
}
DIS_D float2 pmul(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "mul.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
DIS_D float2 bc(float v) { return make_float2(v, v); }

// Coils go two at a time: the pair's X values of one (b, ky) are one float4
// (re, im of coil c, re, im of coil c+1), so a sample's twiddles, its sample
// row and one 16-byte load serve both coils, and the complex products are
// packed f32x2 operations across the pair. The twiddles W2^m sit in shared
// memory; the samples' rows and columns come in CSR order (kyq, kzq), two
// samples per thread and pass so their load and product chains overlap
// (four consecutive positions per thread, sharing a row's loads, measured
// slower: 4.12 against 3.61 ms per forward launch at 256x256x16).

// per sample of the forward sum: (re, im) accumulators of the coil pair and
// the twiddle W2^{kz b} as broadcast pairs, advanced by W2^{kz} per line
struct SumAcc {
  float2 ARp, ARn, AI;  // sum w.x XX, sum w.y XY, sum (w.x XY + w.y XX)
  float2 WX, WY;        // (w.x, w.x), (w.y, w.y)
  float2 SX, SY, SYn;   // step: (s.x, s.x), (s.y, s.y), (-s.y, -s.y)
  int ky;
};

DIS_D void acc_init(SumAcc& A, int ky, int kz, int b0, int N2, const float2* tws) {
  const float2 w = tws[(int)(((long long)kz * b0) % N2)], st = tws[kz];
  A.ARp = A.ARn = A.AI = make_float2(0.f, 0.f);
  A.WX = bc(w.x);
  A.WY = bc(w.y);
  A.SX = bc(st.x);
  A.SY = bc(st.y);
  A.SYn = bc(-st.y);
  A.ky = ky;
}

DIS_D void acc_line(SumAcc& A, const float4 x) {
  const float2 XX = make_float2(x.x, x.z), XY = make_float2(x.y, x.w);
  A.ARp = pfma(A.WX, XX, A.ARp);
  A.ARn = pfma(A.WY, XY, A.ARn);
  A.AI = pfma(A.WX, XY, A.AI);
  A.AI = pfma(A.WY, XX, A.AI);
  const float2 nx = pfma(A.WX, A.SX, pmul(A.WY, A.SYn));
  A.WY = pfma(A.WX, A.SY, pmul(A.WY, A.SX));
  A.WX = nx;
}

// forward: partial sample sums of one (slot, tile of LPB lines along b, n3)
template <int F1, int F2>
__global__ void __launch_bounds__(kThreads) sum_fwd_kernel(SumArgs a, const float2* __restrict__ z,
                                                           const float2* __restrict__ twg) {
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  extern __shared__ __align__(16) float2 sm[];
  float4* Xs = reinterpret_cast<float4*>(sm);  // [LPB][N] coil pairs
  float2* Xh = sm;                             // the same, as (coil, re/im) halves
  float2* tw = sm + 2 * LPB * N;
  float2* ex = tw + LN::TWS;
  float2* tws = ex + LPB * LN::EXSZ;  // W2^m, m < N2
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  for (int m = tid; m < a.N2; m += kThreads) tws[m] = a.tw2[m];
  const int slot = (int)(blockIdx.x % a.n_slots);
  const long long q0 = (long long)(blockIdx.x / a.n_slots) * LPB;  // first line (b + N2 n3)
  const int n3 = (int)(q0 / a.N2), b0 = (int)(q0 % a.N2), tile = b0 / LPB;
  const long long base = (q0 + li) * N;
  float2* myex = ex + li * LN::EXSZ;
  const int seg = a.slot_seg[slot];
  const int* rp = a.rowptr + (long long)seg * (a.N1 + 1);
  const int s0 = rp[0], s1 = rp[a.N1];
  __syncthreads();
  const float2* zs = z + slot * a.Vz;
  float2 zr[F1];
#pragma unroll
  for (int m = 0; m < F1; ++m) zr[m] = lt < F2 ? zs[base + lt + F2 * m] : make_float2(0.f, 0.f);
  for (int c = 0; c < a.C; c += 2) {
    const bool two = c + 1 < a.C;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float2 v[F1], X[F2];
      const float2* S = a.Sf + (c + h) * a.Sc;
      const bool ok = h == 0 || two;
#pragma unroll
      for (int m = 0; m < F1; ++m)
        v[m] = (lt < F2 && ok) ? cmul(S[base + lt + F2 * m], zr[m]) : make_float2(0.f, 0.f);
      LN::fwd(v, X, lt, myex, tw);
      if (lt < F1) {
#pragma unroll
        for (int k2 = 0; k2 < F2; ++k2) Xh[2 * ((long long)li * N + lt + F1 * k2) + h] = X[k2];
      }
      __syncwarp();  // the line's exchange area is reused by the next FFT
    }
    __syncthreads();
    float2* out0 = a.part + ((((long long)slot * a.ntile + tile) * a.C + c) * a.N3c + n3) * a.ldp;
    float2* out1 = out0 + (long long)a.N3c * a.ldp;
    for (int q = s0 + tid; q < s1; q += 2 * kThreads) {
      const int qb = q + kThreads;
      const bool hb = qb < s1;
      SumAcc A, B;
      acc_init(A, a.kyq[q], a.kzq[q], b0, a.N2, tws);
      acc_init(B, hb ? a.kyq[qb] : A.ky, hb ? a.kzq[qb] : 0, b0, a.N2, tws);
#pragma unroll
      for (int j = 0; j < LPB; ++j) {
        acc_line(A, Xs[j * N + A.ky]);
        acc_line(B, Xs[j * N + B.ky]);
      }
      const float2 RA = make_float2(A.ARp.x - A.ARn.x, A.ARp.y - A.ARn.y);
      out0[q - s0] = make_float2(RA.x, A.AI.x);
      if (two) out1[q - s0] = make_float2(RA.y, A.AI.y);
      if (hb) {
        const float2 RB = make_float2(B.ARp.x - B.ARn.x, B.ARp.y - B.ARn.y);
        out0[qb - s0] = make_float2(RB.x, B.AI.x);
        if (two) out1[qb - s0] = make_float2(RB.y, B.AI.y);
      }
    }
    __syncthreads();  // Xs is rewritten by the next coil pair
  }
}

// y[i + ld (n3 + n3off + N3y c)] = scale * sum over tiles of part (- ymeas)
__global__ void sum_reduce_kernel(SumArgs a, float2* __restrict__ y, const float2* __restrict__ ymeas, long long ld,
                                  int n3off, int N3y, float scale) {
  const long long per_slot = (long long)a.C * a.N3c * a.ldp;
  const long long tot = per_slot * a.n_slots;
  const long long ts = (long long)a.C * a.N3c * a.ldp;  // tile stride
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
    const int slot = (int)(e / per_slot);
    const long long r = e % per_slot;  // (c, n3, q)
    const int q = (int)(r % a.ldp);
    const long long cn = r / a.ldp;
    const int n3 = (int)(cn % a.N3c), c = (int)(cn / a.N3c);
    const int seg = a.slot_seg[slot];
    const int* rp = a.rowptr + (long long)seg * (a.N1 + 1);
    if (q >= rp[a.N1] - rp[0]) continue;
    const float2* p = a.part + (long long)slot * a.ntile * ts + r;
    float2 s = make_float2(0.f, 0.f);
    for (int t = 0; t < a.ntile; ++t) s = cadd(s, p[t * ts]);
    const int i = a.perm[rp[0] + q];
    const long long o = i + ld * (n3 + n3off) + ld * N3y * c;
    float2 v = cscale(s, scale);
    if (ymeas) v = csub(v, ymeas[o]);
    y[o] = v;
  }
}

// the adjoint's input: part[slot][c][n3][q - s0] = Mb[n3] We[i] y[i, n3, c]
// for the sample i at CSR position q of the slot's segment (s0 its first)
__global__ void sum_gather_kernel(SumArgs a, const float2* __restrict__ y, long long ld, int n3off, int N3y,
                                  const float* __restrict__ We, const float* __restrict__ Mb) {
  const long long per_slot = (long long)a.C * a.N3c * a.ldp;
  const long long tot = per_slot * a.n_slots;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
    const int slot = (int)(e / per_slot);
    const long long r = e % per_slot;  // (c, n3, k)
    const int k = (int)(r % a.ldp);
    const long long cn = r / a.ldp;
    const int n3 = (int)(cn % a.N3c), c = (int)(cn / a.N3c);
    const int* rp = a.rowptr + (long long)a.slot_seg[slot] * (a.N1 + 1);
    if (k >= rp[a.N1] - rp[0]) continue;
    const int i = a.perm[rp[0] + k];
    float wt = Mb ? Mb[n3 + n3off] : 1.f;
    if (We) wt *= We[i];
    a.part[e] = cscale(y[i + ld * (n3 + n3off) + ld * N3y * c], wt);
  }
}

// adjoint: u[slot] (LPB lines) = scale * sum_c conj(S_c) .* IFFT_1(X_c), X_c
// built from the slot's gathered, weighted samples (sum_gather_kernel)
template <int F1, int F2>
__global__ void __launch_bounds__(kThreads, 2) sum_adj_kernel(SumArgs a, float2* __restrict__ u, float scale,
                                                              const float2* __restrict__ twg) {
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  extern __shared__ __align__(16) float2 sm[];
  float4* Xs = reinterpret_cast<float4*>(sm);  // [LPB][N] coil pairs
  const float2* Xh = sm;                       // the same, as (coil, re/im) halves
  float2* tw = sm + 2 * LPB * N;
  float2* ex = tw + LN::TWS;
  float2* tws = ex + LPB * LN::EXSZ;  // conj(W2^m), m < N2
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  for (int m = tid; m < a.N2; m += kThreads) tws[m] = cconj(a.tw2[m]);
  const int slot = (int)(blockIdx.x % a.n_slots);
  const long long q0 = (long long)(blockIdx.x / a.n_slots) * LPB;
  const int n3 = (int)(q0 / a.N2), b0 = (int)(q0 % a.N2);
  const long long base = (q0 + li) * N;
  float2* myex = ex + li * LN::EXSZ;
  const int seg = a.slot_seg[slot];
  const int* rp = a.rowptr + (long long)seg * (a.N1 + 1);
  __syncthreads();
  float2 acc[F1];
#pragma unroll
  for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
  for (int c = 0; c < a.C; c += 2) {
    const bool two = c + 1 < a.C;
    // this (c, n3) row of the gathered samples, indexed by CSR position
    const float2* yq0 = a.part + (((long long)slot * a.C + c) * a.N3c + n3) * a.ldp - rp[0];
    const float2* yq1 = yq0 + (long long)a.N3c * a.ldp;
    // each row's LPB lines in two halves (rows first, so a warp's stores are
    // consecutive): a thread sums the row's samples into LPB / 2 lines
    constexpr int HL = LPB / 2;
    for (int rr = tid; rr < 2 * a.N1; rr += kThreads) {
      const int r = rr % a.N1, jb = (rr / a.N1) * HL;
      float2 XR[HL], XI[HL];  // lanes: the two coils
#pragma unroll
      for (int j = 0; j < HL; ++j) XR[j] = XI[j] = make_float2(0.f, 0.f);
      const int qe = rp[r + 1];
      for (int q = rp[r]; q < qe; q += 2) {
        // two samples of the row at a time; a missing second one adds zeros
        const bool hb = q + 1 < qe;
        const float2 zero = make_float2(0.f, 0.f);
        const int kz0 = a.kzq[q], kz1 = hb ? a.kzq[q + 1] : kz0;
        const float2 w0 = tws[(int)(((long long)kz0 * (b0 + jb)) % a.N2)], st0 = tws[kz0];
        const float2 w1 = tws[(int)(((long long)kz1 * (b0 + jb)) % a.N2)], st1 = tws[kz1];
        const float2 p0 = cmul(yq0[q], w0);
        const float2 p1 = two ? cmul(yq1[q], w0) : zero;
        const float2 r0 = hb ? cmul(yq0[q + 1], w1) : zero;
        const float2 r1 = (hb && two) ? cmul(yq1[q + 1], w1) : zero;
        float2 VX = make_float2(p0.x, p1.x), VY = make_float2(p0.y, p1.y);
        float2 UX = make_float2(r0.x, r1.x), UY = make_float2(r0.y, r1.y);
        const float2 SX0 = bc(st0.x), SY0 = bc(st0.y), SN0 = bc(-st0.y);
        const float2 SX1 = bc(st1.x), SY1 = bc(st1.y), SN1 = bc(-st1.y);
#pragma unroll
        for (int j = 0; j < HL; ++j) {
          XR[j] = cadd(XR[j], cadd(VX, UX));
          XI[j] = cadd(XI[j], cadd(VY, UY));
          const float2 nx = pfma(VX, SX0, pmul(VY, SN0));
          VY = pfma(VX, SY0, pmul(VY, SX0));
          VX = nx;
          const float2 ux = pfma(UX, SX1, pmul(UY, SN1));
          UY = pfma(UX, SY1, pmul(UY, SX1));
          UX = ux;
        }
      }
#pragma unroll
      for (int j = 0; j < HL; ++j) Xs[(jb + j) * N + r] = make_float4(XR[j].x, XI[j].x, XR[j].y, XI[j].y);
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && !two) break;
      float2 X[F2], v[F1];
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2)
        X[k2] = lt < F1 ? Xh[2 * ((long long)li * N + lt + F1 * k2) + h] : make_float2(0.f, 0.f);
      LN::inv(X, v, lt, myex, tw);
      __syncwarp();
      if (lt < F2) {
        const float2* S = a.Sf + (c + h) * a.Sc + base;
#pragma unroll
        for (int m = 0; m < F1; ++m) acc[m] = cadd(acc[m], cmulc(v[m], S[lt + F2 * m]));
      }
    }
    __syncthreads();  // the next coil pair rewrites Xs
  }
  if (lt < F2) {
    float2* o = u + slot * a.Vz + base;
#pragma unroll
    for (int m = 0; m < F1; ++m) o[lt + F2 * m] = cscale(acc[m], scale);
  }
}

template <int F1, int F2>
struct SumLaunch {
  using LN = ff::Line<F1, F2>;
  static constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  static constexpr int kMaxN2 = 512;  // the shared twiddle table W2^m
  static size_t smem() {
    return sizeof(float2) * (LN::TWS + (size_t)LPB * LN::EXSZ + kMaxN2) + sizeof(float4) * LPB * N;
  }
  static bool init() {
    const int b = (int)smem();
    const int co = (int)cudaSharedmemCarveoutMaxShared;  // two CTAs per SM
    const bool r =
        cudaFuncSetAttribute(sum_fwd_kernel<F1, F2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) == cudaSuccess &&
        cudaFuncSetAttribute(sum_adj_kernel<F1, F2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) == cudaSuccess &&
        cudaFuncSetAttribute(sum_fwd_kernel<F1, F2>, cudaFuncAttributePreferredSharedMemoryCarveout, co) ==
            cudaSuccess &&
        cudaFuncSetAttribute(sum_adj_kernel<F1, F2>, cudaFuncAttributePreferredSharedMemoryCarveout, co) == cudaSuccess;
    cudaGetLastError();
    return r;
  }
  static bool fwd(const SumArgs& a, const float2* z, const float2* tw, cudaStream_t s) {
    static const bool ok = init();
    if (!ok) return false;
    const unsigned grid = (unsigned)(((long long)a.N2 * a.N3c / LPB) * a.n_slots);
    sum_fwd_kernel<F1, F2><<<grid, kThreads, smem(), s>>>(a, z, tw);
    return true;
  }
  static bool adj(const SumArgs& a, float2* u, float scale, const float2* tw, cudaStream_t s) {
    static const bool ok = init();
    if (!ok) return false;
    const unsigned grid = (unsigned)(((long long)a.N2 * a.N3c / LPB) * a.n_slots);
    sum_adj_kernel<F1, F2><<<grid, kThreads, smem(), s>>>(a, u, scale, tw);
    return true;
  }
};

// lines per CTA for a dim-1 length, 0 when no kernel exists
int lines_per_cta(int n1) {
  int F1, F2;
  if (!dis_fast_factor(n1, &F1, &F2)) return 0;
  return kThreads / ff::pow2ceil(F1 > F2 ? F1 : F2);
}

template <class Fn>
bool dispatch(int n1, Fn&& f) {
  switch (n1) {
    case 16: return f(SumLaunch<4, 4>());
    case 32: return f(SumLaunch<8, 4>());
    case 44: return f(SumLaunch<4, 11>());
    case 64: return f(SumLaunch<8, 8>());
    case 88: return f(SumLaunch<8, 11>());
    case 96: return f(SumLaunch<8, 12>());
    case 128: return f(SumLaunch<16, 8>());
    case 160: return f(SumLaunch<16, 10>());
    case 176: return f(SumLaunch<16, 11>());
    case 192: return f(SumLaunch<16, 12>());
    case 256: return f(SumLaunch<16, 16>());
    default: return false;
  }
}

}  // namespace sc

// The sample-sum coil stage runs when the plan's context selects it
// (disorder_ctx_set_tuning), a dim-1 line kernel exists, N2 is a multiple of
// the lines per CTA and the ky rows are at most 4 per thread.
bool dis_sum_coil_usable(const disorder_plan_s* plan) {
  if (!plan->ctx || !plan->ctx->tune_coil || !dis_use_fast()) return false;
  const int lpb = sc::lines_per_cta(plan->N[0]);
  return lpb > 0 && plan->N[1] % lpb == 0 && plan->N[0] <= 4 * fp::kThreads &&
         plan->N[1] <= sc::SumLaunch<16, 16>::kMaxN2;
}

// bytes of partial sums per slot for C coils, N3c readout rows and ldp samples
size_t dis_sum_part_bytes(const disorder_plan_s* plan, int C, int N3c, int ldp) {
  const int lpb = sc::lines_per_cta(plan->N[0]);
  return (size_t)(plan->N[1] / std::max(lpb, 1)) * C * N3c * (size_t)ldp * sizeof(float2);
}

static sc::SumArgs sum_args(const disorder_plan_s* plan, const CoilArgs& a, float2* part, int ldp) {
  sc::SumArgs s;
  s.N1 = a.N1;
  s.N2 = a.N2;
  s.N3c = a.N3c;
  s.Vz = a.Vz;
  s.Sf = a.Sf;
  s.Sc = a.Sc;
  s.C = a.C;
  s.n_slots = a.n_slots;
  s.slot_seg = a.d_slot_seg;
  s.rowptr = plan->d_rowptr;
  s.perm = plan->d_perm;
  s.kyq = plan->d_kyq;
  s.kzq = plan->d_kzq;
  s.tw2 = plan->d_tw[1];
  s.part = part;
  s.ldp = ldp;
  s.ntile = a.N2 / std::max(sc::lines_per_cta(a.N1), 1);
  return s;
}

// encode's coil stage: y (the chunk's slots' samples, rows n3off.. of y) from
// the state volumes z (first readout row of the chunk)
int dis_coil_sum_fwd(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* z,
                     float2* part, int ldp, float2* y, long long y_ld, int y_n3off, int y_N3, const float2* y_meas,
                     float scale) {
  if (a.n_slots == 0 || a.N3c == 0) return DISORDER_OK;
  const sc::SumArgs s = sum_args(plan, a, part, ldp);
  const bool ok = sc::dispatch(a.N1, [&](auto L) { return decltype(L)::fwd(s, z, plan->d_tw[0], ctx->stream); });
  if (!ok) return dis_set_error(ctx, DISORDER_BAD_ARG, "sample-sum coil stage: no kernel for N1=%d", a.N1);
  dis_count(ctx);
  const long long tot = (long long)a.n_slots * a.C * a.N3c * ldp;
  const int blocks = (int)std::min<long long>((tot + 255) / 256, 8LL * ctx->sm_count);
  sc::sum_reduce_kernel<<<std::max(blocks, 1), 256, 0, ctx->stream>>>(s, y, y_meas, y_ld, y_n3off, y_N3, scale);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}

// bytes of the adjoint's gathered samples per slot
size_t dis_sum_gather_bytes(int C, int N3c, int ldq) { return (size_t)C * N3c * (size_t)ldq * sizeof(float2); }

// decode's coil stage: u (slot volumes, first readout row of the chunk) from
// the samples y weighted by We (per sample) and Mb (per readout row); yq:
// dis_sum_gather_bytes per slot of scratch, ldq the most samples of a segment
int dis_coil_sum_adj(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, const float2* y,
                     long long y_ld, int y_n3off, int y_N3, const float* We, const float* Mb, float2* u, float scale,
                     float2* yq, int ldq) {
  if (a.n_slots == 0 || a.N3c == 0) return DISORDER_OK;
  if (!yq || ldq < 1) return dis_set_error(ctx, DISORDER_BAD_ARG, "sample-sum adjoint: no sample scratch");
  const sc::SumArgs s = sum_args(plan, a, yq, ldq);
  const long long tot = (long long)a.n_slots * a.C * a.N3c * ldq;
  const int blocks = (int)std::min<long long>((tot + 255) / 256, 8LL * ctx->sm_count);
  sc::sum_gather_kernel<<<std::max(blocks, 1), 256, 0, ctx->stream>>>(s, y, y_ld, y_n3off, y_N3, We, Mb);
  dis_count(ctx);
  const bool ok = sc::dispatch(a.N1, [&](auto L) { return decltype(L)::adj(s, u, scale, plan->d_tw[0], ctx->stream); });
  if (!ok) return dis_set_error(ctx, DISORDER_BAD_ARG, "sample-sum coil stage: no kernel for N1=%d", a.N1);
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}
