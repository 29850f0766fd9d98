// Fused coil stage: one CTA per (state, readout position) plane.
//
// The encoding of one segment s at readout n3 and coil c is
//   y_i = sum_{n1,n2} F1[ky_i,n1] F2[kz_i,n2] S_c z      (encode.m:120-136)
// with unitary DFT rows. Each shot samples ~1/NS of the ky-kz grid, so instead
// of a full 2-D FFT and a gather we FFT the plane's columns along n1 (all ky
// are used) and evaluate the kz sum only at the segment's samples:
//   y_i = sum_{n2} W_N2^{kz_i n2} X[ky_i, n2],  X = FFT_1(S_c z).
// The adjoint (decode.m:42-58,78-85) rebuilds each column from the samples,
//   X[ky, n2] = sum_{i in row ky} w_i y_i conj(W_N2^{kz_i n2}),
// inverse-FFTs it along n1, multiplies by conj(S_c) and sums over coils in
// registers. The sample values of all coils live in shared memory, so the
// normal operator (encodedecode.m:119-177) needs no intermediate buffers:
// HBM traffic is the state volume, the coil maps (read twice) and the output.
#pragma once
#include "fastfft.cuh"
#include "internal.h"

namespace pl {

constexpr int kThreads = 256;

enum { ENCODE = 0, DECODE = 1, ENCDEC = 2 };

struct PlaneArgs {
  int N1, N2, N3c;          // plane size and readout positions processed
  long long Vz;             // per-slot stride of z (0: one volume shared by all slots)
  long long Vu;             // per-slot stride of u
  const float2* z;          // state volumes (already offset to the first readout)
  float2* u;                // output volumes (DECODE / ENCDEC), same layout as z
  const float2* Sf;         // coil maps (offset to the first readout)
  long long Sc;             // coil stride of Sf
  int C;
  const int* slot_seg;      // segment of each slot
  const long long* seg_off; // sample offsets of the segments
  const int* ky;            // per-sample rows
  const int* kz;
  const int* rowptr;        // per-segment CSR over ky rows (global sample indices)
  const int* perm;
  // samples
  float2* y;                // ENCODE output / DECODE input
  const float2* ymeas;      // ENCODE: subtract (residual) when non-null
  long long ld;             // leading dim of y
  int y_n3off, y_N3;        // readout offset / extent of y's layout
  const float* We;          // per-sample weights or null
  const float* Mb;          // readout weights (DECODE) or null
  float scale_f;            // forward scale (1/sqrt(N1 N2))
  float scale_a;            // adjoint scale
  int max_ns;               // capacity of the sample buffer per coil
};

// shared-memory layout sizes (in float2 units) for a given configuration
template <int F1, int F2>
struct Layout {
  using LN = ff::Line<F1, F2>;
  static constexpr int N1 = LN::N, TL = LN::TL, LPB = kThreads / TL, CB = LPB, XP = CB + 1;
  static size_t bytes(int N2, int C, int max_ns) {
    const size_t f2 = LN::TWS + ((N2 + 1) & ~1) + (size_t)LPB * LN::EXSZ + (size_t)N1 * XP +
                      (size_t)C * max_ns;
    const size_t ints = (size_t)N1 + 1 + 3 * (size_t)max_ns;
    return f2 * sizeof(float2) + ints * sizeof(int) + 64;
  }
};

template <int F1, int F2, int MODE>
__global__ void __launch_bounds__(kThreads) plane_kernel(PlaneArgs a, const float2* __restrict__ tw1g,
                                                         const float2* __restrict__ tw2g) {
  using LY = Layout<F1, F2>;
  using LN = typename LY::LN;
  constexpr int N1 = LY::N1, TL = LY::TL, CB = LY::CB, XP = LY::XP;
  extern __shared__ __align__(16) float2 sm[];
  const int N2 = a.N2;
  float2* tw1 = sm;
  float2* tw2 = tw1 + LN::TWS;
  float2* ex = tw2 + ((N2 + 1) & ~1);
  float2* Xb = ex + LY::LPB * LN::EXSZ;
  float2* yv = Xb + N1 * XP;
  int* s_row = reinterpret_cast<int*>(yv + (size_t)a.C * a.max_ns);  // N1+1 row pointers (local)
  int* s_ky = s_row + N1 + 1;
  int* s_kz = s_ky + a.max_ns;
  int* s_perm = s_kz + a.max_ns;

  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  const int n3 = blockIdx.x, slot = blockIdx.y;
  const int seg = a.slot_seg[slot];
  const long long i0 = a.seg_off[seg];
  const int ns = (int)(a.seg_off[seg + 1] - i0);
  ff::load_tw<F1, F2>(tw1, tw1g, tid, kThreads);
  for (int m = tid; m < N2; m += kThreads) tw2[m] = tw2g[m];
  for (int q = tid; q < ns; q += kThreads) {
    s_ky[q] = a.ky[i0 + q];
    s_kz[q] = a.kz[i0 + q];
  }
  const int* rp = a.rowptr + (long long)seg * (N1 + 1);
  for (int r = tid; r <= N1; r += kThreads) s_row[r] = rp[r] - (int)i0;
  for (int q = tid; q < ns; q += kThreads) s_perm[q] = a.perm[i0 + q] - (int)i0;
  __syncthreads();

  const long long plane = (long long)n3 * N1 * N2;
  const float2* zp = a.z + slot * a.Vz + plane;
  float2* myex = ex + li * LN::EXSZ;

  // ------------------------------------------------------------ forward: sample values of every coil
  if (MODE == ENCODE || MODE == ENCDEC) {
    for (int e = tid; e < a.C * ns; e += kThreads) yv[(e / ns) * a.max_ns + e % ns] = make_float2(0.f, 0.f);
    __syncthreads();
    for (int b0 = 0; b0 < N2; b0 += CB) {
      const int col = b0 + li;
      const bool cv = col < N2;
      float2 zr[F1];
#pragma unroll
      for (int m = 0; m < F1; ++m)
        zr[m] = (cv && lt < F2) ? zp[(long long)col * N1 + lt + F2 * m] : make_float2(0.f, 0.f);
      for (int c = 0; c < a.C; ++c) {
        const float2* S = a.Sf + c * a.Sc + plane + (long long)col * N1;
        float2 v[F1], X[F2];
#pragma unroll
        for (int m = 0; m < F1; ++m) v[m] = (cv && lt < F2) ? cmul(S[lt + F2 * m], zr[m]) : make_float2(0.f, 0.f);
        LN::fwd(v, X, lt, myex, tw1);
        if (lt < F1) {
#pragma unroll
          for (int k2 = 0; k2 < F2; ++k2) Xb[(lt + F1 * k2) * XP + li] = X[k2];
        }
        __syncthreads();
        // each thread owns samples q = tid, tid+256, ...: y_q += sum_j X[ky_q, b0+j] W^{kz_q (b0+j)}
        float2* yc = yv + (size_t)c * a.max_ns;
        const int nc = min(CB, N2 - b0);
        for (int q = tid; q < ns; q += kThreads) {
          const int ky = s_ky[q], kz = s_kz[q];
          int idx = (int)(((long long)kz * b0) % N2);
          float2 acc = yc[q];
          const float2* row = Xb + ky * XP;
          for (int j = 0; j < nc; ++j) {
            acc = cfma(row[j], tw2[idx], acc);
            idx += kz;
            if (idx >= N2) idx -= N2;
          }
          yc[q] = acc;
        }
        __syncthreads();
      }
    }
    if (MODE == ENCODE) {
      for (int e = tid; e < a.C * ns; e += kThreads) {
        const int c = e / ns, q = e % ns;
        const long long gi = a.ld * (n3 + a.y_n3off) + a.ld * a.y_N3 * c + i0 + q;
        float2 v = cscale(yv[(size_t)c * a.max_ns + q], a.scale_f);
        if (a.ymeas) v = csub(v, a.ymeas[gi]);
        a.y[gi] = v;
      }
      return;
    }
    // ENCDEC: weight the samples (the unitary scalings of both directions are in scale_a)
    if (a.We) {
      for (int e = tid; e < a.C * ns; e += kThreads) {
        const int c = e / ns, q = e % ns;
        yv[(size_t)c * a.max_ns + q] = cscale(yv[(size_t)c * a.max_ns + q], a.We[i0 + q]);
      }
    }
    __syncthreads();
  } else {
    // DECODE: sample values from y (times We and Mb)
    const float mb = a.Mb ? a.Mb[n3 + a.y_n3off] : 1.f;
    for (int e = tid; e < a.C * ns; e += kThreads) {
      const int c = e / ns, q = e % ns;
      const long long gi = a.ld * (n3 + a.y_n3off) + a.ld * a.y_N3 * c + i0 + q;
      float w = mb;
      if (a.We) w *= a.We[i0 + q];
      yv[(size_t)c * a.max_ns + q] = cscale(a.y[gi], w);
    }
    __syncthreads();
  }

  // ------------------------------------------------------------ adjoint: columns from samples, inverse FFT, coil sum
  float2* up = a.u + slot * a.Vu + plane;
  for (int b0 = 0; b0 < N2; b0 += CB) {
    const int col = b0 + li;
    const bool cv = col < N2;
    float2 acc[F1];
#pragma unroll
    for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
    const int nc = min(CB, N2 - b0);
    for (int c = 0; c < a.C; ++c) {
      const float2* yc = yv + (size_t)c * a.max_ns;
      // rows owned by threads: X[r, b0+j] = sum_{q in row r} y_q conj(W^{kz_q (b0+j)})
      for (int r = tid; r < N1; r += kThreads) {
        float2 xr[CB];
#pragma unroll
        for (int j = 0; j < CB; ++j) xr[j] = make_float2(0.f, 0.f);
        for (int t = s_row[r]; t < s_row[r + 1]; ++t) {
          const int q = s_perm[t];
          const int kz = s_kz[q];
          const float2 yq = yc[q];
          int idx = (int)(((long long)kz * b0) % N2);
#pragma unroll
          for (int j = 0; j < CB; ++j) {
            xr[j] = cfma(yq, cconj(tw2[idx]), xr[j]);
            idx += kz;
            if (idx >= N2) idx -= N2;
          }
        }
#pragma unroll
        for (int j = 0; j < CB; ++j)
          if (j < nc) Xb[r * XP + j] = xr[j];
      }
      __syncthreads();
      float2 X[F2], v[F1];
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) X[k2] = (cv && lt < F1) ? Xb[(lt + F1 * k2) * XP + li] : make_float2(0.f, 0.f);
      __syncthreads();
      LN::inv(X, v, lt, myex, tw1);
      if (cv && lt < F2) {
        const float2* S = a.Sf + c * a.Sc + plane + (long long)col * N1;
#pragma unroll
        for (int m = 0; m < F1; ++m) acc[m] = cadd(acc[m], cmulc(v[m], S[lt + F2 * m]));
      }
    }
    if (cv && lt < F2) {
#pragma unroll
      for (int m = 0; m < F1; ++m) up[(long long)col * N1 + lt + F2 * m] = cscale(acc[m], a.scale_a);
    }
  }
}

template <int F1, int F2>
struct PlaneLaunch {
  static bool run(int mode, const PlaneArgs& a, const float2* tw1, const float2* tw2, int n_slots,
                  cudaStream_t s) {
    const size_t smem = Layout<F1, F2>::bytes(a.N2, a.C, a.max_ns);
    if (smem > 225 * 1024) return false;
    static bool once = [] {
      cudaFuncSetAttribute(plane_kernel<F1, F2, ENCODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 226 * 1024);
      cudaFuncSetAttribute(plane_kernel<F1, F2, DECODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 226 * 1024);
      cudaFuncSetAttribute(plane_kernel<F1, F2, ENCDEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, 226 * 1024);
      return true;
    }();
    (void)once;
    dim3 grid((unsigned)a.N3c, (unsigned)n_slots);
    if (mode == ENCODE)
      plane_kernel<F1, F2, ENCODE><<<grid, kThreads, smem, s>>>(a, tw1, tw2);
    else if (mode == DECODE)
      plane_kernel<F1, F2, DECODE><<<grid, kThreads, smem, s>>>(a, tw1, tw2);
    else
      plane_kernel<F1, F2, ENCDEC><<<grid, kThreads, smem, s>>>(a, tw1, tw2);
    return true;
  }
};

}  // namespace pl
