// Line-pass kernels on the register-resident FFT engine (fastfft.cuh).
// Included by the fast_*.cu instantiation units; see fastpass.h for the
// host-side launchers.
#pragma once
#include "fastfft.cuh"
#include "internal.h"

namespace fp {

constexpr int kThreads = 256;

DIS_D int even(int n) { return (n + 1) & ~1; }

// Line geometry of a pass along `axis` of an N0 x N1 x N2 volume for the
// thread's line: line li of the tile. Axis-0 tiles are LPB consecutive
// contiguous lines; axis-1/2 tiles are LPB lines adjacent along axis 0.
struct LineInfo {
  long long base;
  int coord[3];
  bool valid;
};

DIS_D LineInfo line_info(const int* N, int axis, int lpb, int tile, int li) {
  LineInfo r;
  r.coord[0] = r.coord[1] = r.coord[2] = 0;
  if (axis == 0) {
    const long long q = (long long)tile * lpb + li;
    r.valid = q < (long long)N[1] * N[2];
    if (r.valid) {
      r.coord[1] = (int)(q % N[1]);
      r.coord[2] = (int)(q / N[1]);
    }
    r.base = r.valid ? q * N[0] : 0;
  } else {
    const int nt0 = (N[0] + lpb - 1) / lpb;
    const int other = tile / nt0;
    const int c0 = (tile % nt0) * lpb + li;
    r.valid = c0 < N[0];
    if (r.valid) {
      r.coord[0] = c0;
      r.coord[axis == 1 ? 2 : 1] = other;
    }
    r.base = !r.valid ? 0
                      : (axis == 1 ? c0 + (long long)other * N[0] * N[1] : c0 + (long long)other * N[0]);
  }
  return r;
}

// First element of tile `tile` for strided passes (line 0 of the tile) and
// the number of valid lines in it.
DIS_D void strided_tile(const int* N, int axis, int lpb, int tile, long long* base0, int* nvalid) {
  const int nt0 = (N[0] + lpb - 1) / lpb;
  const int other = tile / nt0;
  const int c0 = (tile % nt0) * lpb;
  *nvalid = min(lpb, N[0] - c0);
  *base0 = axis == 1 ? c0 + (long long)other * N[0] * N[1] : c0 + (long long)other * N[0];
}

DIS_D long long axis_stride(const int* N, int axis) {
  return axis == 0 ? 1LL : (axis == 1 ? (long long)N[0] : (long long)N[0] * N[1]);
}

// staged tile load: st[p*(LPB+1) + l] = src[base0 + l + p*stride] for l < nvalid.
// Fully unrolled with all global loads issued before the shared stores so
// that every thread keeps IT loads in flight.
template <int N, int LPB>
DIS_D void stage_load(const float2* __restrict__ src, float2* st, long long base0, long long stride, int nvalid,
                      int tid) {
  constexpr int TOT = N * LPB, IT = (TOT + kThreads - 1) / kThreads;
  float2 v[IT];
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int e = tid + it * kThreads;
    const int p = e / LPB, l = e % LPB;
    v[it] = (e < TOT && l < nvalid) ? src[base0 + l + p * stride] : make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int e = tid + it * kThreads;
    if (e < TOT) st[(e / LPB) * (LPB + 1) + e % LPB] = v[it];
  }
}

template <int N, int LPB>
DIS_D void stage_store(float2* __restrict__ dst, const float2* st, long long base0, long long stride, int nvalid,
                       int tid) {
  constexpr int TOT = N * LPB, IT = (TOT + kThreads - 1) / kThreads;
#pragma unroll
  for (int it = 0; it < IT; ++it) {
    const int e = tid + it * kThreads;
    const int p = e / LPB, l = e % LPB;
    if (e < TOT && l < nvalid) dst[base0 + l + p * stride] = st[p * (LPB + 1) + l];
  }
}

// coefficient of code `code` at frequency k, given the slot's table rows
template <class LN>
DIS_D float2 coefB(int code, const float2* tA, const float2* tB, const float* kG, int k) {
  switch (code) {
    case P_A:
      return tA[k];
    case P_B:
      return tB[k];
    case P_ONE:
      return make_float2(1.0f / LN::N, 0.f);
    case P_DK:
      return make_float2(0.f, -kG[k] * (1.0f / LN::N));
    default:
      return make_float2(0.f, 0.f);
  }
}

// ---------------------------------------------------------------- transform pass
// MODE bit 0: a second input and/or output (gradient passes); bit 1: sum
// the output over the slots (last pass of the inverse transform).
template <int F1, int F2, int MODE>
__global__ void __launch_bounds__(kThreads) line_kernel(LinePassArgs a, const float2* __restrict__ twg) {
  constexpr bool DUAL = (MODE & 1) != 0, ACC = (MODE & 2) != 0;
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  float2* ex = sm + LN::TWS;
  float2* st = ex + LPB * LN::EXSZ;
  const int tid = threadIdx.x;
  const int lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  const LineInfo L = line_info(a.N, a.axis, LPB, blockIdx.x, li);
  const int rowA = a.A.b == 0 ? L.coord[0] : (a.A.b == 1 ? L.coord[1] : (a.A.b == 2 ? L.coord[2] : 0));
  const int rowB = a.B.b == 0 ? L.coord[0] : (a.B.b == 1 ? L.coord[1] : (a.B.b == 2 ? L.coord[2] : 0));
  const bool staged = a.axis != 0;
  long long sbase = 0;
  int snv = 0;
  const long long sstr = axis_stride(a.N, a.axis);
  if (staged) strided_tile(a.N, a.axis, LPB, blockIdx.x, &sbase, &snv);
  float2* myex = ex + li * LN::EXSZ;
  __syncthreads();
  const bool two_in = DUAL && a.in1 != nullptr, two_out = DUAL && a.out1 != nullptr;
  float2 acc[F1];
#pragma unroll
  for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
  int s_begin = blockIdx.y, s_end = blockIdx.y + 1;
  if (ACC) {
    s_begin = 0;
    s_end = a.n_slots;
  }
  for (int slot = s_begin; slot < s_end; ++slot) {
    float2 a0[F1], a1[F1], c0[F2], c1[F2];
    // ---- load (layout A)
    const float2* in0 = a.in0 + slot * a.in0_s;
    const float2* in1 = two_in ? a.in1 + slot * a.in1_s : nullptr;
    if (!staged) {
#pragma unroll
      for (int m = 0; m < F1; ++m) {
        a0[m] = (L.valid && lt < F2) ? in0[L.base + lt + F2 * m] : make_float2(0.f, 0.f);
        if (two_in) a1[m] = (L.valid && lt < F2) ? in1[L.base + lt + F2 * m] : make_float2(0.f, 0.f);
      }
    } else {
      stage_load<N, LPB>(in0, st, sbase, sstr, snv, tid);
      __syncthreads();
#pragma unroll
      for (int m = 0; m < F1; ++m) a0[m] = lt < F2 ? st[(lt + F2 * m) * (LPB + 1) + li] : make_float2(0.f, 0.f);
      __syncthreads();
      if (two_in) {
        stage_load<N, LPB>(in1, st, sbase, sstr, snv, tid);
        __syncthreads();
#pragma unroll
        for (int m = 0; m < F1; ++m) a1[m] = lt < F2 ? st[(lt + F2 * m) * (LPB + 1) + li] : make_float2(0.f, 0.f);
        __syncthreads();
      }
    }
    // ---- forward FFT(s)
    LN::fwd(a0, c0, lt, myex, tw);
    if (two_in) LN::fwd(a1, c1, lt, myex, tw);
    // ---- combine in frequency, in place (layout B: k = lt + F1*k2)
    if (!two_in) {
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) c1[k2] = make_float2(0.f, 0.f);
    }
    if (lt < F1) {
      const float2* tA = a.A.p ? a.A.p + slot * a.A.sstride + (long long)rowA * N : nullptr;
      const float2* tB = a.B.p ? a.B.p + slot * a.B.sstride + (long long)rowB * N : nullptr;
      const float2* tT = a.T.p ? a.T.p + slot * a.T.sstride : nullptr;
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) {
        const int k = lt + F1 * k2;
        const float2 x0 = c0[k2];
        const float2 x1 = c1[k2];
        float2 v0 = cmul(coefB<LN>(a.c00, tA, tB, a.kG, k), x0);
        if (a.c01) v0 = cadd(v0, cmul(coefB<LN>(a.c01, tA, tB, a.kG, k), x1));
        float2 v1 = make_float2(0.f, 0.f);
        if (two_out) {
          v1 = cmul(coefB<LN>(a.c10, tA, tB, a.kG, k), x0);
          if (a.c11) v1 = cadd(v1, cmul(coefB<LN>(a.c11, tA, tB, a.kG, k), x1));
        }
        if (tT) {
          const float2 tf = tT[k];
          v0 = cmul(v0, tf);
          v1 = cmul(v1, tf);
        }
        c0[k2] = v0;
        c1[k2] = v1;
      }
    }
    // ---- inverse FFT(s) back to layout A
    LN::inv(c0, a0, lt, myex, tw);
    if (two_out) LN::inv(c1, a1, lt, myex, tw);
    // ---- store
    if (ACC) {
#pragma unroll
      for (int m = 0; m < F1; ++m) acc[m] = cadd(acc[m], a0[m]);
    } else if (!staged) {
      float2* o0 = a.out0 + slot * a.out0_s;
      float2* o1 = two_out ? a.out1 + slot * a.out1_s : nullptr;
      if (L.valid && lt < F2) {
#pragma unroll
        for (int m = 0; m < F1; ++m) {
          o0[L.base + lt + F2 * m] = a0[m];
          if (two_out) o1[L.base + lt + F2 * m] = a1[m];
        }
      }
    } else {
      if (lt < F2) {
#pragma unroll
        for (int m = 0; m < F1; ++m) st[(lt + F2 * m) * (LPB + 1) + li] = a0[m];
      }
      __syncthreads();
      stage_store<N, LPB>(a.out0 + slot * a.out0_s, st, sbase, sstr, snv, tid);
      __syncthreads();
      if (two_out) {
        if (lt < F2) {
#pragma unroll
          for (int m = 0; m < F1; ++m) st[(lt + F2 * m) * (LPB + 1) + li] = a1[m];
        }
        __syncthreads();
        stage_store<N, LPB>(a.out1 + slot * a.out1_s, st, sbase, sstr, snv, tid);
        __syncthreads();
      }
    }
  }
  if (ACC) {
    const float beta = a.beta;
    if (!staged) {
      if (L.valid && lt < F2) {
#pragma unroll
        for (int m = 0; m < F1; ++m) {
          const long long g = L.base + lt + F2 * m;
          float2 v = acc[m];
          if (beta != 0.f) v = cadd(v, cscale(a.out0[g], beta));
          a.out0[g] = v;
        }
      }
    } else {
      if (lt < F2) {
#pragma unroll
        for (int m = 0; m < F1; ++m) st[(lt + F2 * m) * (LPB + 1) + li] = acc[m];
      }
      __syncthreads();
      for (int e = tid; e < N * LPB; e += kThreads) {
        const int p = e / LPB, l = e % LPB;
        if (l < snv) {
          const long long g = sbase + l + p * sstr;
          float2 v = st[p * (LPB + 1) + l];
          if (beta != 0.f) v = cadd(v, cscale(a.out0[g], beta));
          a.out0[g] = v;
        }
      }
    }
  }
}

// ---------------------------------------------------------------- coil stage, axis 0 (length N1 = F1*F2)
// expand: A[slot][c] = FFT_1(S_c .* z[slot]) stored in natural frequency order.
template <int F1, int F2>
__global__ void __launch_bounds__(kThreads) expand_kernel(CoilArgs a, const float2* __restrict__ z,
                                                          float2* __restrict__ A, const float2* __restrict__ twg) {
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  float2* ex = sm + LN::TWS;
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  const long long nlines = (long long)a.N2 * a.N3c;
  // 1-D grid with the slot fastest: the CTAs of all slots of one tile run
  // together and read that tile's coil-map lines once from HBM, then from L2
  const int slot = (int)(blockIdx.x % a.n_slots);
  const long long q = (long long)(blockIdx.x / a.n_slots) * LPB + li;
  const bool valid = q < nlines && lt < F2;
  const long long base = q * N;
  float2* myex = ex + li * LN::EXSZ;
  __syncthreads();
  const float2* zs = z + slot * a.Vz;
  float2 zr[F1];
#pragma unroll
  for (int m = 0; m < F1; ++m) zr[m] = valid ? zs[base + lt + F2 * m] : make_float2(0.f, 0.f);
  const long long Vc = nlines * N;
  for (int c = 0; c < a.C; ++c) {
    const float2* S = a.Sf + c * a.Sc;
    float2 v[F1], X[F2];
#pragma unroll
    for (int m = 0; m < F1; ++m) v[m] = valid ? cmul(S[base + lt + F2 * m], zr[m]) : make_float2(0.f, 0.f);
    LN::fwd(v, X, lt, myex, tw);
    if (q < nlines && lt < F1) {
      float2* o = A + ((long long)slot * a.C + c) * Vc + base;
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) o[lt + F1 * k2] = X[k2];
    }
  }
}

// combine: u[slot] = scale * sum_c conj(S_c) .* IFFT_1(A[slot][c])
template <int F1, int F2>
__global__ void __launch_bounds__(kThreads) combine_kernel(CoilArgs a, const float2* __restrict__ A,
                                                           float2* __restrict__ u, float scale,
                                                           const float2* __restrict__ twg) {
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  float2* ex = sm + LN::TWS;
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  const long long nlines = (long long)a.N2 * a.N3c;
  // 1-D grid with the slot fastest (coil-map lines shared through L2)
  const int slot = (int)(blockIdx.x % a.n_slots);
  const long long q = (long long)(blockIdx.x / a.n_slots) * LPB + li;
  const bool ok = q < nlines;
  const long long base = q * N;
  float2* myex = ex + li * LN::EXSZ;
  __syncthreads();
  const long long Vc = nlines * N;
  float2 acc[F1];
#pragma unroll
  for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
  for (int c = 0; c < a.C; ++c) {
    const float2* src = A + ((long long)slot * a.C + c) * Vc + base;
    float2 X[F2], v[F1];
#pragma unroll
    for (int k2 = 0; k2 < F2; ++k2) X[k2] = (ok && lt < F1) ? src[lt + F1 * k2] : make_float2(0.f, 0.f);
    LN::inv(X, v, lt, myex, tw);
    if (ok && lt < F2) {
      const float2* S = a.Sf + c * a.Sc + base;
#pragma unroll
      for (int m = 0; m < F1; ++m) acc[m] = cadd(acc[m], cmulc(v[m], S[lt + F2 * m]));
    }
  }
  if (ok && lt < F2) {
    float2* o = u + slot * a.Vz + base;
#pragma unroll
    for (int m = 0; m < F1; ++m) o[lt + F2 * m] = cscale(acc[m], scale);
  }
}

// ---------------------------------------------------------------- coil stage, axis 1 (length N2 = F1*F2)
// Tiles: LPB consecutive ky rows (axis 0) at fixed readout n3 of one
// (slot, coil) volume of the N1 x N2 x N3c slab.
struct Tile1 {
  int ky0, n3, nl;
};

template <int LPB>
DIS_D Tile1 tile1(int N1, int tile) {
  const int nt0 = (N1 + LPB - 1) / LPB;
  Tile1 t;
  t.n3 = tile / nt0;
  t.ky0 = (tile % nt0) * LPB;
  t.nl = min(LPB, N1 - t.ky0);
  return t;
}

// mode 0: gather samples (encode), 1: weight map (encodedecode), 2: scatter (decode)
template <int F1, int F2, int MODE>
__global__ void __launch_bounds__(kThreads) axis1_kernel(CoilArgs a, float2* __restrict__ A, float2* __restrict__ y,
                                                         const float2* __restrict__ ymeas, long long ld, int n3off,
                                                         int N3y, float scale, const float* __restrict__ wmap,
                                                         const float* __restrict__ We, const float* __restrict__ Mb,
                                                         const int* __restrict__ rowptr,
                                                         const int* __restrict__ perm, const int* __restrict__ kyv,
                                                         const int* __restrict__ kzv, const float2* __restrict__ twg) {
  using LN = ff::Line<F1, F2>;
  constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL, P = LPB + 1;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  float2* ex = sm + LN::TWS;
  float2* st = ex + LPB * LN::EXSZ;
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  const int N1 = a.N1;
  const Tile1 t = tile1<LPB>(N1, blockIdx.x);
  const int c = blockIdx.y, slot = blockIdx.z;
  const long long Vc = (long long)N1 * N * a.N3c;
  float2* vol = A + ((long long)slot * a.C + c) * Vc + t.ky0 + (long long)t.n3 * N1 * N;
  float2* myex = ex + li * LN::EXSZ;
  const int seg = a.d_slot_seg[slot];
  const int* rp = rowptr + (long long)seg * (N1 + 1);
  float2 v[F1], X[F2];
  if (MODE == 2) {
    for (int e = tid; e < N * P; e += kThreads) st[e] = make_float2(0.f, 0.f);
    __syncthreads();
    const int s0 = rp[t.ky0], s1 = rp[t.ky0 + t.nl];
    const long long ib = ld * (t.n3 + n3off) + ld * N3y * c;
    const float mb = Mb ? Mb[t.n3 + n3off] : 1.f;
    for (int qq = s0 + tid; qq < s1; qq += kThreads) {
      const int i = perm[qq];
      float w = mb;
      if (We) w *= We[i];
      const float2 val = cscale(y[ib + i], w);
      float2* d = &st[kzv[i] * P + (kyv[i] - t.ky0)];
      atomicAdd(&d->x, val.x);
      atomicAdd(&d->y, val.y);
    }
    __syncthreads();
#pragma unroll
    for (int k2 = 0; k2 < F2; ++k2) X[k2] = lt < F1 ? st[(lt + F1 * k2) * P + li] : make_float2(0.f, 0.f);
    __syncthreads();
  } else {
    stage_load<N, LPB>(vol, st, 0, N1, t.nl, tid);
    __syncthreads();
#pragma unroll
    for (int m = 0; m < F1; ++m) v[m] = lt < F2 ? st[(lt + F2 * m) * P + li] : make_float2(0.f, 0.f);
    __syncthreads();
    LN::fwd(v, X, lt, myex, tw);
  }
  if (MODE == 0) {
    if (lt < F1) {
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) st[(lt + F1 * k2) * P + li] = X[k2];
    }
    __syncthreads();
    const int s0 = rp[t.ky0], s1 = rp[t.ky0 + t.nl];
    const long long ob = ld * (t.n3 + n3off) + ld * N3y * c;
    for (int qq = s0 + tid; qq < s1; qq += kThreads) {
      const int i = perm[qq];
      float2 val = cscale(st[kzv[i] * P + (kyv[i] - t.ky0)], scale);
      if (ymeas) val = csub(val, ymeas[ob + i]);
      y[ob + i] = val;
    }
    return;
  }
  if (MODE == 1) {
    const float* wm = wmap + ((long long)seg * N1 + t.ky0 + li) * N;
    if (lt < F1) {
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) {
        const float w = li < t.nl ? wm[lt + F1 * k2] : 0.f;
        X[k2] = cscale(X[k2], w);
      }
    }
  }
  LN::inv(X, v, lt, myex, tw);
  if (lt < F2) {
#pragma unroll
    for (int m = 0; m < F1; ++m) st[(lt + F2 * m) * P + li] = v[m];
  }
  __syncthreads();
  stage_store<N, LPB>(vol, st, 0, N1, t.nl, tid);
}

// ---------------------------------------------------------------- launchers
template <class K>
void smem_attr(K k) {
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

template <int F1, int F2>
struct Launch {
  using LN = ff::Line<F1, F2>;
  static constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  static size_t smem(bool staged) {
    return sizeof(float2) * (LN::TWS + LPB * LN::EXSZ + (staged ? (size_t)N * (LPB + 1) : 0));
  }
  static bool init() {
    smem_attr(line_kernel<F1, F2, 0>);
    smem_attr(line_kernel<F1, F2, 1>);
    smem_attr(line_kernel<F1, F2, 2>);
    smem_attr(expand_kernel<F1, F2>);
    smem_attr(combine_kernel<F1, F2>);
    smem_attr(axis1_kernel<F1, F2, 0>);
    smem_attr(axis1_kernel<F1, F2, 1>);
    smem_attr(axis1_kernel<F1, F2, 2>);
    return true;
  }
  static void line(const LinePassArgs& a, const float2* tw, cudaStream_t s) {
    static bool once = init();
    (void)once;
    size_t tiles;
    if (a.axis == 0)
      tiles = ((size_t)a.N[1] * a.N[2] + LPB - 1) / LPB;
    else
      tiles = (size_t)((a.N[0] + LPB - 1) / LPB) * (a.axis == 1 ? a.N[2] : a.N[1]);
    dim3 grid((unsigned)tiles, a.accumulate ? 1u : (unsigned)a.n_slots);
    const size_t sm = smem(a.axis != 0);
    if (a.accumulate)
      line_kernel<F1, F2, 2><<<grid, kThreads, sm, s>>>(a, tw);
    else if (a.in1 || a.out1)
      line_kernel<F1, F2, 1><<<grid, kThreads, sm, s>>>(a, tw);
    else
      line_kernel<F1, F2, 0><<<grid, kThreads, sm, s>>>(a, tw);
  }
  static void expand(const CoilArgs& a, const float2* z, float2* A, const float2* tw, cudaStream_t s) {
    static bool once = init();
    (void)once;
    const long long nl = (long long)a.N2 * a.N3c;
    const unsigned grid = (unsigned)(((nl + LPB - 1) / LPB) * a.n_slots);
    expand_kernel<F1, F2><<<grid, kThreads, smem(false), s>>>(a, z, A, tw);
  }
  static void combine(const CoilArgs& a, const float2* A, float2* u, float scale, const float2* tw, cudaStream_t s) {
    static bool once = init();
    (void)once;
    const long long nl = (long long)a.N2 * a.N3c;
    const unsigned grid = (unsigned)(((nl + LPB - 1) / LPB) * a.n_slots);
    combine_kernel<F1, F2><<<grid, kThreads, smem(false), s>>>(a, A, u, scale, tw);
  }
  static void axis1(int mode, const CoilArgs& a, float2* A, float2* y, const float2* ymeas, long long ld, int n3off,
                    int N3y, float scale, const float* wmap, const float* We, const float* Mb,
                    const disorder_plan_s* plan, const float2* tw, cudaStream_t s) {
    static bool once = init();
    (void)once;
    dim3 grid((unsigned)(((a.N1 + LPB - 1) / LPB) * a.N3c), (unsigned)a.C, (unsigned)a.n_slots);
    const size_t sm = smem(true);
    if (mode == 0)
      axis1_kernel<F1, F2, 0><<<grid, kThreads, sm, s>>>(a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb,
                                                         plan->d_rowptr, plan->d_perm, plan->d_ky, plan->d_kz, tw);
    else if (mode == 1)
      axis1_kernel<F1, F2, 1><<<grid, kThreads, sm, s>>>(a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb,
                                                         plan->d_rowptr, plan->d_perm, plan->d_ky, plan->d_kz, tw);
    else
      axis1_kernel<F1, F2, 2><<<grid, kThreads, sm, s>>>(a, A, y, ymeas, ld, n3off, N3y, scale, wmap, We, Mb,
                                                         plan->d_rowptr, plan->d_perm, plan->d_ky, plan->d_kz, tw);
  }
};

}  // namespace fp

#define DIS_FAST_INSTANTIATE(F1, F2) template struct fp::Launch<F1, F2>;
