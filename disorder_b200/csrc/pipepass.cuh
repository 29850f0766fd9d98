// Pipelined single-input transform pass on the register-resident FFT engine.
//
// The line passes of the sinc rigid transform (one DFT along an axis, a
// per-frequency phase, one inverse DFT) stream every element through HBM
// once in and once out. The one-tile-per-CTA kernel in fastpass.cuh issues a
// tile's loads, waits for them, and only then transforms, so each SM has
// little memory traffic in flight. Here a persistent CTA walks a sequence of
// (tile, slot) items and stages each tile in shared memory with 16-byte
// cp.async copies, double-buffered: the copy of item j+1 is in flight while
// item j is transformed. The stage buffer of the current item doubles as the
// FFT exchange area once its data sit in registers, which keeps a CTA at
// about 72 KB of shared memory for N = 256 (three CTAs per SM).
//
// Covers the passes with one input and one output (the forward and inverse
// transform and the translation passes); the dual-volume gradient passes
// keep the kernel in fastpass.cuh.
#pragma once
#include "fastpass.cuh"

namespace fp {

DIS_D void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
DIS_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
DIS_D void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
DIS_D void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Element (p, l) of a strided-tile stage buffer: rows p of LPB elements, the
// 16-byte chunks (element pairs) of row p XOR-permuted by p mod 8, so that
// the reads of layout A (16 rows, 2 adjacent columns per warp) and the
// row-wise copies both take the minimum number of shared-memory wavefronts.
template <int LPB>
DIS_D int swz(int p, int l) {
  return p * LPB + (((((l >> 1) ^ (p & 7)) & (LPB / 2 - 1)) << 1) | (l & 1));
}

template <int F1, int F2>
struct Pipe {
  using LN = ff::Line<F1, F2>;
  static constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL, TILE = N * LPB;
  static constexpr int EXT = LPB * LN::EXSZ;
  static constexpr int SB = ((TILE > EXT ? TILE : EXT) + 1) & ~1;  // one stage buffer, float2
  static constexpr int TW = (N + 1) & ~1;                          // twiddles, float2
  static constexpr size_t SMEM = sizeof(float2) * (TW + 2 * (size_t)SB);
  static_assert(LPB >= 16, "the chunk swizzle needs at least 8 chunks per row");
};

// ACC: out0 = beta*out0 + sum over the slots (each CTA owns whole tiles and
// walks their slots in order); otherwise out0[slot] = pass(in0[slot]).
// SEED: the coefficient of frequency k = lt + F1*k2 is generated from the
// line's row of phase seeds (a.Sd, tables.cu seed_table_kernel) as
// lo[lt]*step^k2 for the non-negative frequencies and hi[lt]*step^(k2-k2h)
// for the negative ones, instead of being loaded from the A and T tables.
template <int F1, int F2, bool ACC, bool SEED>
__global__ void __launch_bounds__(kThreads, ACC ? 2 : 3) pipe_kernel(LinePassArgs a, const float2* __restrict__ twg,
                                                                     int n_tiles) {
  using P = Pipe<F1, F2>;
  using LN = typename P::LN;
  constexpr int N = P::N, TL = P::TL, LPB = P::LPB, TILE = P::TILE, SB = P::SB;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  float2* stg = sm + P::TW;
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  for (int m = tid; m < N; m += kThreads) tw[m] = twg[m];
  const int axis = a.axis, S = a.n_slots, G = gridDim.x, b = blockIdx.x;
  const long long sstr = axis_stride(a.N, axis);
  const long long nlines0 = (long long)a.N[1] * a.N[2];
  // n_tiles * S < 2^31 (checked on the host)
  int n_items;
  if (ACC)
    n_items = b < n_tiles ? ((n_tiles - 1 - b) / G + 1) * S : 0;
  else {
    const int nw = n_tiles * S;
    n_items = b < nw ? (nw - 1 - b) / G + 1 : 0;
  }
  // item j of this CTA -> (tile, slot); without ACC the items are tile-major
  // over the grid so that a shared input (in0_s == 0) is re-read from L2
  auto item = [&](int j, int& tile, int& slot) {
    if (ACC) {
      tile = b + (j / S) * G;
      slot = j % S;
    } else {
      const int w = b + j * G;
      tile = w / S;
      slot = w % S;
    }
  };
  auto issue = [&](int j, float2* st) {
    int tile, slot;
    item(j, tile, slot);
    const float2* src = a.in0 + slot * a.in0_s;
    if (axis == 0) {
      const long long q0 = (long long)tile * LPB;
      const int nl = (int)min((long long)LPB, nlines0 - q0);
      const float2* g = src + q0 * N;
      const int chunks = nl * (N / 2);
#pragma unroll 1
      for (int c = tid; c < chunks; c += kThreads) cp_async16(st + 2 * c, g + 2 * c);
    } else {
      long long base0;
      int nv;
      strided_tile(a.N, axis, LPB, tile, &base0, &nv);
      const int cpr = nv >> 1;  // nv is even: N0 is even and tiles start at multiples of LPB
      constexpr int CH = N * (LPB / 2);
#pragma unroll 1
      for (int c = tid; c < CH; c += kThreads) {
        const int p = c / (LPB / 2), k = c % (LPB / 2);
        if (k < cpr) cp_async16(st + swz<LPB>(p, 2 * k), src + base0 + 2 * k + p * sstr);
      }
    }
  };

  float2 acc[F1];
#pragma unroll
  for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
  if (n_items > 0) issue(0, stg);
  cp_async_commit();
  for (int j = 0; j < n_items; ++j) {
    float2* st = stg + (j & 1) * SB;
    if (j + 1 < n_items) issue(j + 1, stg + ((j + 1) & 1) * SB);
    cp_async_commit();
    int tile, slot;
    item(j, tile, slot);
    const LineInfo L = line_info(a.N, axis, LPB, tile, li);
    // phase seeds of this line, loaded while the tile lands
    float2 slo, shi, sst;
    if (SEED && lt < F1) {
      const int row = a.Sd.b == 0 ? L.coord[0] : (a.Sd.b == 1 ? L.coord[1] : (a.Sd.b == 2 ? L.coord[2] : 0));
      const float2* sr = a.Sd.p + slot * a.Sd.sstride + row * a.sd_w;
      slo = sr[lt];
      shi = sr[F1 + lt];
      sst = sr[2 * F1];
    }
    cp_async_wait_1();
    __syncthreads();  // item j staged; twiddles visible
    long long base0 = 0;
    int nv = 0;
    if (axis != 0) strided_tile(a.N, axis, LPB, tile, &base0, &nv);
    float2 v[F1], X[F2];
#pragma unroll
    for (int m = 0; m < F1; ++m) {
      const int p = lt + F2 * m;
      float2 e = make_float2(0.f, 0.f);
      if (lt < F2 && L.valid) e = axis == 0 ? st[li * N + p] : st[swz<LPB>(p, li)];
      v[m] = e;
    }
    __syncthreads();  // the stage buffer becomes the exchange area
    float2* myex = st + li * LN::EXSZ;
    LN::fwd(v, X, lt, myex, tw);
    if (SEED && lt < F1) {
      constexpr int KP = F2 / 2;             // k2 < KP: k < N/2 for every lt
      constexpr bool ODD = (F2 & 1) != 0;    // odd F2: k2 == KP straddles N/2 at lt = F1/2
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) {
        float2 c;
        if (k2 < KP) {
          c = slo;
          if (k2 + 1 < KP || ODD) slo = cmul(slo, sst);
        } else if (ODD && k2 == KP) {
          c = (2 * lt < F1) ? slo : cmul(shi, cconj(sst));
        } else {
          c = shi;
          if (k2 + 1 < F2) shi = cmul(shi, sst);
        }
        X[k2] = cmul(c, X[k2]);
      }
    } else if (!SEED && lt < F1) {
      const int rowA = a.A.b == 0 ? L.coord[0] : (a.A.b == 1 ? L.coord[1] : (a.A.b == 2 ? L.coord[2] : 0));
      const float2* tA = a.A.p ? a.A.p + slot * a.A.sstride + (long long)rowA * N : nullptr;
      const float2* tT = a.T.p ? a.T.p + slot * a.T.sstride : nullptr;
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) {
        const int k = lt + F1 * k2;
        float2 c = coefB<LN>(a.c00, tA, nullptr, a.kG, k);
        if (tT) c = cmul(c, tT[k]);
        X[k2] = cmul(c, X[k2]);
      }
    }
    LN::inv(X, v, lt, myex, tw);
    if (ACC) {
#pragma unroll
      for (int m = 0; m < F1; ++m) acc[m] = cadd(acc[m], v[m]);
      if (slot == S - 1) {
        const float beta = a.beta;
        if (axis == 0) {
          if (L.valid && lt < F2) {
#pragma unroll
            for (int m = 0; m < F1; ++m) {
              const long long g = L.base + lt + F2 * m;
              float2 o = acc[m];
              if (beta != 0.f) o = cadd(o, cscale(a.out0[g], beta));
              a.out0[g] = o;
            }
          }
        } else {
          __syncthreads();  // every line's exchange is done
          if (lt < F2 && L.valid) {
#pragma unroll
            for (int m = 0; m < F1; ++m) st[swz<LPB>(lt + F2 * m, li)] = acc[m];
          }
          __syncthreads();
          for (int e = tid; e < TILE; e += kThreads) {
            const int p = e / LPB, l = e % LPB;
            if (l < nv) {
              const long long g = base0 + l + p * sstr;
              float2 o = st[swz<LPB>(p, l)];
              if (beta != 0.f) o = cadd(o, cscale(a.out0[g], beta));
              a.out0[g] = o;
            }
          }
        }
#pragma unroll
        for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
      }
    } else if (axis == 0) {
      float2* o0 = a.out0 + slot * a.out0_s;
      if (L.valid && lt < F2) {
#pragma unroll
        for (int m = 0; m < F1; ++m) o0[L.base + lt + F2 * m] = v[m];
      }
    } else {
      __syncthreads();  // every line's exchange is done
      if (lt < F2 && L.valid) {
#pragma unroll
        for (int m = 0; m < F1; ++m) st[swz<LPB>(lt + F2 * m, li)] = v[m];
      }
      __syncthreads();
      float2* o0 = a.out0 + slot * a.out0_s;
      constexpr int IT = (TILE + kThreads - 1) / kThreads;
#pragma unroll 4
      for (int it = 0; it < IT; ++it) {
        const int e = tid + it * kThreads;
        const int p = e / LPB, l = e % LPB;
        if (e < TILE && l < nv) o0[base0 + l + p * sstr] = st[swz<LPB>(p, l)];
      }
    }
    __syncthreads();  // the buffer is free for the copy issued by the next item
  }
  cp_async_wait_0();
}

template <int F1, int F2>
struct PipeLaunch {
  using P = Pipe<F1, F2>;
  struct Occ {
    int per_sm[4] = {0, 0, 0, 0};  // [acc + 2*seed]
    int sms = 0;
  };
  template <bool ACC, bool SEED>
  static void prep(Occ& o) {
    auto k = pipe_kernel<F1, F2, ACC, SEED>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per_sm[(ACC ? 1 : 0) + (SEED ? 2 : 0)], k, kThreads, P::SMEM);
  }
  static Occ init() {
    Occ o;
    prep<false, false>(o);
    prep<true, false>(o);
    prep<false, true>(o);
    prep<true, true>(o);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev);
    return o;
  }
  // Whether the pass fits this kernel: one input, one output, coefficient
  // A (or a constant) times the optional T row, 16-byte aligned slots, even N0.
  static bool eligible(const LinePassArgs& a) {
    if (a.in1 || a.out1 || a.c01 != P_ZERO || a.c00 == P_B) return false;
    if ((a.N[0] & 1) || (reinterpret_cast<uintptr_t>(a.in0) & 15) || (a.in0_s & 1)) return false;
    return true;
  }
  static bool run(const LinePassArgs& a, const float2* tw, cudaStream_t s) {
    static const Occ occ = init();
    if (!eligible(a)) return false;
    const int acc = a.accumulate ? 1 : 0;
    const bool seed = a.Sd.p != nullptr && a.sd_w == 2 * F1 + 2 && (a.c00 == P_A || a.c00 == P_ONE);
    const int var = acc + (seed ? 2 : 0);
    if (occ.per_sm[var] <= 0 || occ.sms <= 0) return false;
    long long tiles;
    if (a.axis == 0)
      tiles = ((long long)a.N[1] * a.N[2] + P::LPB - 1) / P::LPB;
    else
      tiles = (long long)((a.N[0] + P::LPB - 1) / P::LPB) * (a.axis == 1 ? a.N[2] : a.N[1]);
    if (tiles * a.n_slots >= (1LL << 31)) return false;
    const long long units = acc ? tiles : tiles * a.n_slots;
    const long long cap = (long long)occ.sms * occ.per_sm[var];
    const unsigned grid = (unsigned)(units < cap ? units : cap);
    const int nt = (int)tiles;
    switch (var) {
      case 0: pipe_kernel<F1, F2, false, false><<<grid, kThreads, P::SMEM, s>>>(a, tw, nt); break;
      case 1: pipe_kernel<F1, F2, true, false><<<grid, kThreads, P::SMEM, s>>>(a, tw, nt); break;
      case 2: pipe_kernel<F1, F2, false, true><<<grid, kThreads, P::SMEM, s>>>(a, tw, nt); break;
      default: pipe_kernel<F1, F2, true, true><<<grid, kThreads, P::SMEM, s>>>(a, tw, nt); break;
    }
    return true;
  }
};

}  // namespace fp

#define DIS_PIPE_INSTANTIATE(F1, F2) template struct fp::PipeLaunch<F1, F2>;
