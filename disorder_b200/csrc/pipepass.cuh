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
DIS_D void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
DIS_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
DIS_D void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
DIS_D void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Stage buffers are line-major: line l of the tile occupies
// [l*pitch, l*pitch + N), and the same span (EXSZ <= pitch) is that line's
// FFT exchange area once its data sit in registers, so a line's lanes only
// synchronise among themselves (__syncwarp) between the two uses.
//   axis 0:   pitch PL (even): each line is copied as 16-byte chunks;
//   axis 1/2: pitch PS (odd): a tile row (one element of each line) is
//             copied as 8-byte elements, and both the copies (consecutive
//             lines, stride PS) and the FFT reads (consecutive elements of
//             one line) hit distinct bank pairs.
template <int F1, int F2>
struct Pipe {
  using LN = ff::Line<F1, F2>;
  static constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  static constexpr int LEN = N > LN::EXSZ ? N : LN::EXSZ;
  static constexpr int PL = (LEN + 1) & ~1, PS = LEN | 1;
  static constexpr int SB = (LPB * (PL > PS ? PL : PS) + 1) & ~1;  // one stage buffer, float2
  static constexpr int TW = LN::TWS;                               // twiddles, float2 (even)
  static constexpr size_t SMEM = sizeof(float2) * (TW + 2 * (size_t)SB);
  // strided copies: RS rows of the tile per sweep of the CTA
  static constexpr int RS = kThreads / LPB, SWEEPS = (N + RS - 1) / RS;
  static_assert(kThreads % LPB == 0, "whole rows per sweep");
};

// One work item of a CTA: tile `tile` of slot `slot` and the tile's geometry
// (32-bit: the volume holds fewer than 2^31 elements, checked on the host).
//   axis 0:   lines q0 .. q0+nv-1 (q = n1 + N1*n2), base = q0*N0, (ca, cb) = (n1, n2) of line q0
//   axis 1/2: lines n0 = ca .. ca+nv-1 at the other coordinate cb, base = first element
struct PItem {
  int tile, slot, base, nv, ca, cb;
};

DIS_D PItem pitem(const int* N, int axis, int lpb, int tile, int slot) {
  PItem it;
  it.tile = tile;
  it.slot = slot;
  if (axis == 0) {
    const int q0 = tile * lpb;
    it.nv = min(lpb, N[1] * N[2] - q0);
    it.base = q0 * N[0];
    it.cb = q0 / N[1];
    it.ca = q0 - it.cb * N[1];
  } else {
    const int nt0 = (N[0] + lpb - 1) / lpb;
    it.cb = tile / nt0;
    it.ca = (tile - it.cb * nt0) * lpb;
    it.nv = min(lpb, N[0] - it.ca);
    it.base = axis == 1 ? it.ca + it.cb * N[0] * N[1] : it.ca + it.cb * N[0];
  }
  return it;
}

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
  constexpr int N = P::N, TL = P::TL, LPB = P::LPB, SB = P::SB, PL = P::PL, PS = P::PS, RS = P::RS;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  float2* stg = sm + P::TW;
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  const int axis = a.axis, S = a.n_slots, G = gridDim.x, b = blockIdx.x;
  const int sstr = axis == 0 ? 1 : (axis == 1 ? a.N[0] : a.N[0] * a.N[1]);
  // n_tiles * S < 2^31 (checked on the host)
  int n_items;
  if (ACC)
    n_items = b < n_tiles ? ((n_tiles - 1 - b) / G + 1) * S : 0;
  else {
    const int nw = n_tiles * S;
    n_items = b < nw ? (nw - 1 - b) / G + 1 : 0;
  }
  if (n_items == 0) return;
  // Item j of this CTA: with ACC, tile b + (j / S)*G and slot j % S; without,
  // w = b + j*G, tile w / S and slot w % S (tile-major over the grid, so a
  // shared input, in0_s == 0, is re-read from L2). Advanced incrementally.
  const int gq = ACC ? 0 : G / S, gr = ACC ? 0 : G % S;
  auto advance = [&](const PItem& c) {
    int tile = c.tile, slot = c.slot;
    if (ACC) {
      if (++slot == S) {
        slot = 0;
        tile += G;
      }
    } else {
      slot += gr;
      tile += gq;
      if (slot >= S) {
        slot -= S;
        ++tile;
      }
    }
    return pitem(a.N, axis, LPB, tile, slot);
  };
  // strided copies: this thread moves line sl, rows sp0 + RS*i
  const int sl = tid % LPB, sp0 = tid / LPB;
  auto issue = [&](const PItem& it, float2* st) {
    const float2* src = a.in0 + it.slot * a.in0_s + it.base;
    if (axis == 0) {
      constexpr int CPL = N / 2, CH = LPB * CPL, IT = (CH + kThreads - 1) / kThreads;
      if (it.nv == LPB) {
#pragma unroll
        for (int i = 0; i < IT; ++i) {
          const int c = tid + i * kThreads;
          const int l = c / CPL, o = c - l * CPL;
          if (CH % kThreads == 0 || c < CH) cp_async16(st + l * PL + 2 * o, src + 2 * c);
        }
      } else {
        const int chunks = it.nv * CPL;
#pragma unroll 1
        for (int c = tid; c < chunks; c += kThreads) {
          const int l = c / CPL, o = c - l * CPL;
          cp_async16(st + l * PL + 2 * o, src + 2 * c);
        }
      }
    } else if (sl < it.nv) {
      const float2* g = src + sl + sp0 * sstr;
      float2* d = st + sl * PS + sp0;
#pragma unroll
      for (int i = 0; i < P::SWEEPS; ++i)
        if (N % RS == 0 || sp0 + RS * i < N) cp_async8(d + RS * i, g + (long long)RS * i * sstr);
    }
  };

  float2 acc[F1];
#pragma unroll
  for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
  PItem cur = pitem(a.N, axis, LPB, ACC ? b : b / S, ACC ? 0 : b % S);
  issue(cur, stg);
  cp_async_commit();
  for (int j = 0; j < n_items; ++j) {
    float2* st = stg + (j & 1) * SB;
    // this thread's line of the current item
    const bool valid = li < cur.nv;
    int c0 = 0, c1 = 0, c2 = 0;
    if (axis == 0) {
      c1 = cur.ca + li;
      c2 = cur.cb;
      while (c1 >= a.N[1]) {
        c1 -= a.N[1];
        ++c2;
      }
    } else {
      c0 = cur.ca + li;
      if (axis == 1)
        c2 = cur.cb;
      else
        c1 = cur.cb;
    }
    // phase seeds of this line, loaded while the tile lands
    float2 slo, shi, sst;
    if (SEED && lt < F1) {
      const int row = a.Sd.b == 0 ? c0 : (a.Sd.b == 1 ? c1 : (a.Sd.b == 2 ? c2 : 0));
      const float2* sr = a.Sd.p + cur.slot * a.Sd.sstride + (valid ? row : 0) * a.sd_w;
      slo = sr[lt];
      shi = sr[F1 + lt];
      sst = sr[2 * F1];
    }
    cp_async_wait_0();
    // item j staged (and twiddles visible); every thread is past item j-1,
    // so the other buffer is free for the next item's copy
    __syncthreads();
    PItem nxt = cur;
    if (j + 1 < n_items) {
      nxt = advance(cur);
      issue(nxt, stg + ((j + 1) & 1) * SB);
    }
    cp_async_commit();
    float2* my = st + li * (axis == 0 ? PL : PS);
    float2 v[F1], X[F2];
#pragma unroll
    for (int m = 0; m < F1; ++m) v[m] = (lt < F2 && valid) ? my[lt + F2 * m] : make_float2(0.f, 0.f);
    __syncwarp();  // the line's span becomes its exchange area
    LN::fwd(v, X, lt, my, tw);
    if (SEED && lt < F1) {
      constexpr int KP = F2 / 2;           // k2 < KP: k < N/2 for every lt
      constexpr bool ODD = (F2 & 1) != 0;  // odd F2: k2 == KP straddles N/2 at lt = F1/2
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
      const int rowA = a.A.b == 0 ? c0 : (a.A.b == 1 ? c1 : (a.A.b == 2 ? c2 : 0));
      const float2* tA = a.A.p ? a.A.p + cur.slot * a.A.sstride + (long long)(valid ? rowA : 0) * N : nullptr;
      const float2* tT = a.T.p ? a.T.p + cur.slot * a.T.sstride : nullptr;
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) {
        const int k = lt + F1 * k2;
        float2 c = coefB<LN>(a.c00, tA, nullptr, a.kG, k);
        if (tT) c = cmul(c, tT[k]);
        X[k2] = cmul(c, X[k2]);
      }
    }
    LN::inv(X, v, lt, my, tw);
    const bool last = !ACC || cur.slot == S - 1;
    if (ACC) {
#pragma unroll
      for (int m = 0; m < F1; ++m) acc[m] = cadd(acc[m], v[m]);
      if (last) {
#pragma unroll
        for (int m = 0; m < F1; ++m) v[m] = acc[m];
#pragma unroll
        for (int m = 0; m < F1; ++m) acc[m] = make_float2(0.f, 0.f);
      }
    }
    if (last) {
      float2* o0 = a.out0 + (ACC ? 0 : cur.slot * a.out0_s) + cur.base;
      const float beta = ACC ? a.beta : 0.f;
      if (axis == 0) {
        // element lt + F2*m of this line, straight from registers
        if (valid && lt < F2) {
          float2* ol = o0 + li * N + lt;
#pragma unroll
          for (int m = 0; m < F1; ++m) {
            float2 o = v[m];
            if (ACC && beta != 0.f) o = cadd(o, cscale(ol[F2 * m], beta));
            ol[F2 * m] = o;
          }
        }
      } else {
        // back into the line's span, then tile rows as 16-byte pairs of lines
        if (lt < F2) {
#pragma unroll
          for (int m = 0; m < F1; ++m) my[lt + F2 * m] = v[m];
        }
        __syncthreads();
        constexpr int PPR = LPB / 2, RO = kThreads / PPR;  // line pairs per row, rows per sweep
        const int q = tid % PPR, r0 = tid / PPR;
        if (2 * q < cur.nv) {  // nv is even: N0 is even and tiles start at multiples of LPB
          const float2* s0 = st + 2 * q * PS + r0;
          float2* g = o0 + 2 * q + (long long)r0 * sstr;
#pragma unroll
          for (int i = 0; i < (N + RO - 1) / RO; ++i) {
            if (N % RO == 0 || r0 + RO * i < N) {
              const float2 e0 = s0[RO * i], e1 = s0[RO * i + PS];
              float4 o = make_float4(e0.x, e0.y, e1.x, e1.y);
              float4* gp = reinterpret_cast<float4*>(g + (long long)RO * i * sstr);
              if (ACC && beta != 0.f) {
                const float4 w = *gp;
                o.x += beta * w.x;
                o.y += beta * w.y;
                o.z += beta * w.z;
                o.w += beta * w.w;
              }
              *gp = o;
            }
          }
        }
      }
    }
    cur = nxt;
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
    cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
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
  // Whether the pass fits this kernel: one input, one output, coefficient A
  // (or a constant) times the optional T row, 16-byte aligned volumes, even
  // N0 and fewer than 2^31 elements per volume.
  static bool eligible(const LinePassArgs& a) {
    if (a.in1 || a.out1 || a.c01 != P_ZERO || a.c00 == P_B) return false;
    if ((a.N[0] & 1) || (long long)a.N[0] * a.N[1] * a.N[2] >= (1LL << 31)) return false;
    if ((reinterpret_cast<uintptr_t>(a.in0) & 15) || (a.in0_s & 1)) return false;
    if ((reinterpret_cast<uintptr_t>(a.out0) & 15) || (a.out0_s & 1)) return false;
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

// ---------------------------------------------------------------- weighted pass of the normal operator
// A[slot][c] <- IFFT_2(w_seg .* FFT_2(A[slot][c])) in place (unnormalised;
// the combine step applies the scale), the dim-2 step of encodedecode on the
// per-coil intermediates of an N1 x N2 x N3c slab (ky fastest). w_seg is the
// segment's sample-weight map wmap[seg][ky][kz]. Work unit = (tile of LPB ky
// rows at one readout position, slot); the CTA walks the unit's C coils with
// the same double-buffered pipeline as pipe_kernel (strided layout), so the
// unit's weights come from L1 after its first coil.
template <int F1, int F2>
__global__ void __launch_bounds__(kThreads, 3) wpipe_kernel(CoilArgs a, float2* __restrict__ A,
                                                            const float* __restrict__ wmap,
                                                            const float2* __restrict__ twg, int n_tiles) {
  using P = Pipe<F1, F2>;
  using LN = typename P::LN;
  constexpr int N = P::N, TL = P::TL, LPB = P::LPB, SB = P::SB, PS = P::PS, RS = P::RS;
  extern __shared__ __align__(16) float2 sm[];
  float2* tw = sm;
  float2* stg = sm + P::TW;
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  const int Nv[3] = {a.N1, a.N2, a.N3c};
  const int S = a.n_slots, C = a.C, G = gridDim.x, b = blockIdx.x;
  const int sstr = a.N1;
  const long long Vc = (long long)a.N1 * a.N2 * a.N3c;
  // units u = b + i*G < n_tiles*S (tile u / S, slot u % S), C items each
  const int nu = n_tiles * S;
  const int n_items = b < nu ? ((nu - 1 - b) / G + 1) * C : 0;
  if (n_items == 0) return;
  const int gq = G / S, gr = G % S;
  auto unit_item = [&](int tile, int slot) { return pitem(Nv, 1, LPB, tile, slot); };
  auto vol = [&](const PItem& it, int c) { return A + ((long long)it.slot * C + c) * Vc + it.base; };
  const int sl = tid % LPB, sp0 = tid / LPB;
  auto issue = [&](const PItem& it, int c, float2* st) {
    if (sl < it.nv) {
      const float2* g = vol(it, c) + sl + sp0 * sstr;
      float2* d = st + sl * PS + sp0;
#pragma unroll
      for (int i = 0; i < P::SWEEPS; ++i)
        if (N % RS == 0 || sp0 + RS * i < N) cp_async8(d + RS * i, g + (long long)RS * i * sstr);
    }
  };
  PItem cur = unit_item(b / S, b % S);
  int cc = 0;
  issue(cur, 0, stg);
  cp_async_commit();
  for (int j = 0; j < n_items; ++j) {
    float2* st = stg + (j & 1) * SB;
    const bool valid = li < cur.nv;
    // the line's weights w[seg][ky = ca + li][kz] (the same for all C coils of
    // the unit, so read from L1 after the first coil)
    const float* wm = wmap + ((long long)a.d_slot_seg[cur.slot] * a.N1 + cur.ca + (valid ? li : 0)) * a.N2;
    cp_async_wait_0();
    __syncthreads();  // item j staged; every thread is past item j-1
    PItem nxt = cur;
    int cn = cc + 1;
    if (j + 1 < n_items) {
      if (cn == C) {
        cn = 0;
        int slot = cur.slot + gr, tile = cur.tile + gq;
        if (slot >= S) {
          slot -= S;
          ++tile;
        }
        nxt = unit_item(tile, slot);
      }
      issue(nxt, cn, stg + ((j + 1) & 1) * SB);
    }
    cp_async_commit();
    float2* my = st + li * PS;
    float2 v[F1], X[F2];
#pragma unroll
    for (int m = 0; m < F1; ++m) v[m] = (lt < F2 && valid) ? my[lt + F2 * m] : make_float2(0.f, 0.f);
    __syncwarp();  // the line's span becomes its exchange area
    LN::fwd(v, X, lt, my, tw);
    if (lt < F1) {
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) X[k2] = cscale(X[k2], wm[lt + F1 * k2]);
    }
    LN::inv(X, v, lt, my, tw);
    if (lt < F2) {
#pragma unroll
      for (int m = 0; m < F1; ++m) my[lt + F2 * m] = v[m];
    }
    __syncthreads();
    constexpr int PPR = LPB / 2, RO = kThreads / PPR;  // line pairs per row, rows per sweep
    const int q = tid % PPR, r0 = tid / PPR;
    if (2 * q < cur.nv) {  // nv is even: N1 is even and tiles start at multiples of LPB
      const float2* s0 = st + 2 * q * PS + r0;
      float2* g = vol(cur, cc) + 2 * q + (long long)r0 * sstr;
#pragma unroll
      for (int i = 0; i < (N + RO - 1) / RO; ++i) {
        if (N % RO == 0 || r0 + RO * i < N) {
          const float2 e0 = s0[RO * i], e1 = s0[RO * i + PS];
          *reinterpret_cast<float4*>(g + (long long)RO * i * sstr) = make_float4(e0.x, e0.y, e1.x, e1.y);
        }
      }
    }
    cur = nxt;
    cc = cn;
  }
  cp_async_wait_0();
}

template <int F1, int F2>
struct WPipeLaunch {
  using P = Pipe<F1, F2>;
  struct Occ {
    int per_sm = 0, sms = 0;
  };
  static Occ init() {
    Occ o;
    cudaFuncSetAttribute(wpipe_kernel<F1, F2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::SMEM);
    cudaFuncSetAttribute(wpipe_kernel<F1, F2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per_sm, wpipe_kernel<F1, F2>, kThreads, P::SMEM);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev);
    return o;
  }
  // false when the slab does not fit this kernel (odd N1, unaligned A,
  // 2^31 or more units)
  static bool run(const CoilArgs& a, float2* A, const float* wmap, const float2* tw, cudaStream_t s) {
    static const Occ occ = init();
    if (occ.per_sm <= 0 || occ.sms <= 0) return false;
    if ((a.N1 & 1) || (reinterpret_cast<uintptr_t>(A) & 15)) return false;
    if ((long long)a.N1 * a.N2 * a.N3c >= (1LL << 31)) return false;
    const long long tiles = (long long)((a.N1 + P::LPB - 1) / P::LPB) * a.N3c;
    const long long units = tiles * a.n_slots;
    if (units == 0 || units * a.C >= (1LL << 31)) return false;
    const long long cap = (long long)occ.sms * occ.per_sm;
    const unsigned grid = (unsigned)(units < cap ? units : cap);
    wpipe_kernel<F1, F2><<<grid, kThreads, P::SMEM, s>>>(a, A, wmap, tw, (int)tiles);
    return true;
  }
};

}  // namespace fp

#define DIS_PIPE_INSTANTIATE(F1, F2) \
  template struct fp::PipeLaunch<F1, F2>; \
  template struct fp::WPipeLaunch<F1, F2>;
