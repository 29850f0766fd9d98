// Mixed-precision line pass of the sinc rigid transform: the DFTs along a
// strided axis as tensor-core GEMMs (tcgen05, BF16x3 or 3xTF32, FP32
// accumulation in tensor memory).
//
// The reference applies every 1-D DFT as a matrix product along one dimension
// (Methods/fftGPU.m:37-43, ifftGPU.m:31-42 through matfun / pagefun). Here a
// line of N = 16 * F2 points (N = 256 or 176) is transformed by the four-step
// factorisation n = t + F2 m, k = k1 + 16 k2, each step a small GEMM over the
// lines of a tile of 16 lines:
//   stage 1  a[l,t][k1] = sum_m W_16^{m k1} x_l[t + F2 m]          (K = m)
//            a[l,t][k1] *= W_N^{t k1}                              (twiddle)
//   stage 2  X_l[k1 + 16 k2] = sum_t W_F2^{t k2} a[l,t][k1]         (K = t)
//            X_l[k] *= c_l[k]      (the pass's phase factor, 1/N folded in)
//   stage 3  z[l,k1][t] = sum_k2 W_F2^{-k2 t} X_l[k1 + 16 k2]       (K = k2)
//            z[l,k1][t] *= W_N^{-t k1}
//   stage 4  y_l[t + F2 m] = sum_k1 W_16^{-k1 m} z[l,k1][t]         (K = k1)
// Complex products are real GEMMs over (index, re/im): A rows are (line,
// index) pairs (16 x 16 = 256 rows, two M = 128 MMAs), K = 32 (16 complex,
// F2 = 11 padded with zeros), B is the 32 x 32 real block form of the small
// DFT matrix, N = 32. The per-line phase factors come from the same per-row
// seeds as the CUDA-core pass (tables.cu), in the same frequency order.
//
// Operands: every product is split into two tensor-core parts (BF16x3: bf16
// hi + lo; 3xTF32: tf32 hi + lo) and hi*hi + hi*lo + lo*hi is accumulated in
// FP32. Rows of every operand follow rho(l, u) = 32 grp + lane with
// lane = (l & 7) + 8 (u & 3) and grp = (l >> 3) + 2 (u >> 2), so the two
// transposing steps (stage 1 -> 2 and 3 -> 4), where a thread scatters its
// row's 16 values into 16 rows, hit 32 distinct banks per warp.
//
// Stages 3 and 4 use the conjugate DFT matrices; they run as the forward
// matrices of stages 2 and 1 on conjugated operands (conj(W^-1 v) =
// W conj(v)), so one 32 x 32 block serves all four stages when F2 = 16 and
// two blocks (W_16, W_F2) when F2 = 11.
//
// Threads: 256; thread (warp w, lane i) owns accumulator row
// 128 (w >> 2) + 32 (w & 3) + i, i.e. line l = (i & 7) + 8 (w & 1) and index
// u = (i >> 3) + 8 (w >> 2) + 4 ((w >> 1) & 1), reading tensor-memory lanes of
// its warp's quadrant. Tiles move by TMA as in tmapass.cuh (no cluster
// multicast, this GPU's buffers only) through one stage buffer: the next
// tile's load is issued as soon as stage 1 has read the current one, and the
// result is staged for its TMA store in the operand area, free after stage 4.
// That keeps a CTA at 72 KB (BF16x3) or 107 KB (3xTF32) of shared memory,
// three or two CTAs per SM, whose stages overlap one another's waits. Every
// wait is bounded and a wait that runs out sets the error word, drains the
// copies in flight, frees the tensor memory and stops the CTA.
#include <cuda_bf16.h>

#include "tmapass.cuh"
#include "umma.cuh"

namespace {

using fp::PItem;
using fp::TArgs;

constexpr int kUT = 256;
constexpr uint32_t kMmaWait = 1u << 20;

template <int F2, bool TF32>
struct UCfg {
  static constexpr int N = 16 * F2;
  static constexpr int ES = TF32 ? 4 : 2;                // operand element bytes
  static constexpr int KSTEP = TF32 ? 8 : 16;
  static constexpr int KS = 32 / KSTEP;                  // MMAs along K per product
  static constexpr int ABYTES = 256 * 32 * ES;           // one part of A
  static constexpr int BBYTES = 32 * 32 * ES;            // one part of one B
  static constexpr int TILE = 16 * N;                    // float2 per tile
  static constexpr int SBB = ((8 * TILE) + 1023) & ~1023;
  // distinct DFT blocks: W_16 (stages 1, 4) and W_F2 (stages 2, 3), one when F2 = 16
  static constexpr int NBM = F2 == 16 ? 1 : 2;
  static constexpr size_t SMEM = 1024 + (size_t)SBB + 2 * ABYTES + 2 * NBM * BBYTES + 8 * 16 * F2;
  static constexpr int MIN_CTAS = TF32 ? 2 : 3;
  static_assert(8 * TILE <= 2 * ABYTES, "the result tile is staged in the operand area");
};

DIS_D int rho(int l, int u) { return 32 * ((l >> 3) + 2 * (u >> 2)) + (l & 7) + 8 * (u & 3); }

// byte offset of element (r, k) of an R-row K-major operand
template <bool TF32>
DIS_D uint32_t opo(int r, int k, int R) {
  constexpr int ES = TF32 ? 4 : 2, E = 16 / ES;
  return (uint32_t)((k / E) * (R * 16) + r * 16 + (k % E) * ES);
}

// store the complex pair (re, im) at K columns (2j, 2j+1) of row r
template <bool TF32>
DIS_D void put_pair(unsigned char* hi, unsigned char* lo, int r, int R, int j, float2 v) {
  const uint32_t o = opo<TF32>(r, 2 * j, R);
  if (TF32) {
    float h0, l0, h1, l1;
    um::split_tf32(v.x, h0, l0);
    um::split_tf32(v.y, h1, l1);
    *reinterpret_cast<float2*>(hi + o) = make_float2(h0, h1);
    *reinterpret_cast<float2*>(lo + o) = make_float2(l0, l1);
  } else {
    uint32_t h, l;
    um::split_bf16x2(v.x, v.y, h, l);
    *reinterpret_cast<uint32_t*>(hi + o) = h;
    *reinterpret_cast<uint32_t*>(lo + o) = l;
  }
}

// a whole row of 16 complex values (K = 32), written in 16-byte pieces
template <bool TF32>
DIS_D void put_row(unsigned char* hi, unsigned char* lo, int r, const float2 (&v)[16]) {
  if (TF32) {
#pragma unroll
    for (int c = 0; c < 16; c += 2) {  // 2 complex (4 fp32) per 16-byte chunk
      float h[4], l[4];
      um::split_tf32(v[c].x, h[0], l[0]);
      um::split_tf32(v[c].y, h[1], l[1]);
      um::split_tf32(v[c + 1].x, h[2], l[2]);
      um::split_tf32(v[c + 1].y, h[3], l[3]);
      const uint32_t o = opo<true>(r, 2 * c, 256);
      *reinterpret_cast<float4*>(hi + o) = make_float4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<float4*>(lo + o) = make_float4(l[0], l[1], l[2], l[3]);
    }
  } else {
#pragma unroll
    for (int c = 0; c < 16; c += 4) {  // 4 complex (8 bf16) per 16-byte chunk
      uint32_t h[4], l[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) um::split_bf16x2(v[c + q].x, v[c + q].y, h[q], l[q]);
      const uint32_t o = opo<false>(r, 2 * c, 256);
      *reinterpret_cast<uint4*>(hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  }
}

// the 32 accumulator columns of this thread's row as 16 complex values
DIS_D void row_load(uint32_t taddr, float2 (&v)[16]) {
  float a[16], b[16];
  um::tld16(taddr, a);
  um::tld16(taddr + 16, b);
  um::tld_wait();
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = make_float2(a[2 * j], a[2 * j + 1]);
    v[8 + j] = make_float2(b[2 * j], b[2 * j + 1]);
  }
}

template <int F2, bool TF32>
__global__ void __launch_bounds__(kUT, (UCfg<F2, TF32>::MIN_CTAS))
    umma_line_kernel(const __grid_constant__ CUtensorMap in_map, const __grid_constant__ CUtensorMap out_map,
                     TArgs t, const float2* __restrict__ twg, int n_tiles, int shared_input) {
  using U = UCfg<F2, TF32>;
  constexpr int N = U::N;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ uint64_t tbar;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tbase;
  const uint32_t base_s = um::saddr(smraw);
  unsigned char* al = smraw + (((base_s + 1023u) & ~1023u) - base_s);
  float2* st = reinterpret_cast<float2*>(al);
  unsigned char* Ahi = al + U::SBB;
  unsigned char* Alo = Ahi + U::ABYTES;
  float2* res = reinterpret_cast<float2*>(Ahi);  // the result tile, after stage 4
  unsigned char* Bm = Alo + U::ABYTES;  // [block][part] blocks of BBYTES
  float2* tws = reinterpret_cast<float2*>(Bm + 2 * U::NBM * U::BBYTES);  // [t][k1] = W_N^{t k1}
  const int tid = threadIdx.x, w = tid >> 5, i = tid & 31;
  const int ml = (i & 7) + 8 * (w & 1);                      // this thread's line
  const int mu = (i >> 3) + 8 * (w >> 2) + 4 * ((w >> 1) & 1);  // this thread's index (t or k1)
  const int myrow = rho(ml, mu);

  // ---- constant operands: the 32 x 32 real DFT blocks, and twiddles
  for (int e = tid; e < U::NBM * 32 * 32; e += kUT) {
    const int blk = e / 1024, n = (e / 32) % 32, k = e % 32;
    const int jo = n >> 1, ro = n & 1, ji = k >> 1, ri = k & 1;
    float2 W = make_float2(0.f, 0.f);
    if (blk == 0) W = twg[(F2 * ji * jo) % N];                            // W_16^{m k1} (symmetric)
    if (blk == 1 && jo < F2 && ji < F2) W = twg[(16 * ji * jo) % N];      // W_F2^{t k2} (symmetric)
    const float val = ro == 0 ? (ri == 0 ? W.x : -W.y) : (ri == 0 ? W.y : W.x);
    unsigned char* hb = Bm + (2 * blk) * U::BBYTES;
    unsigned char* lb = hb + U::BBYTES;
    const uint32_t o = opo<TF32>(n, k, 32);
    if (TF32) {
      float h, l;
      um::split_tf32(val, h, l);
      *reinterpret_cast<float*>(hb + o) = h;
      *reinterpret_cast<float*>(lb + o) = l;
    } else {
      const __nv_bfloat16 h = __float2bfloat16_rn(val);
      const __nv_bfloat16 l = __float2bfloat16_rn(val - __bfloat162float(h));
      *reinterpret_cast<__nv_bfloat16*>(hb + o) = h;
      *reinterpret_cast<__nv_bfloat16*>(lb + o) = l;
    }
  }
  for (int e = tid; e < 16 * F2; e += kUT) tws[e] = twg[((e / 16) * (e % 16)) % N];
  if (tid == 0) {
    um::bar_init(&tbar, 1);
    um::bar_init(&mbar, 1);
    fp::fence_async_smem();
  }
  if (w == 0) {
    um::tmem_alloc(&tbase, 64);
    um::tmem_relinquish();
  }
  um::fence_smem_async();
  um::fence_before_sync();
  __syncthreads();
  um::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t trow = tmem + ((uint32_t)(32 * (w & 3)) << 16) + 32 * (w >> 2);  // this thread's D row
  const uint32_t idd = um::idesc(TF32 ? um::kTF32 : um::kBF16, 128, 32);

  // ---- item walk (as tma_kernel KIND 0)
  const int G = gridDim.x, b = blockIdx.x;
  const int S = t.n_vol;
  const int nu = n_tiles * S;
  const int n_items = b < nu ? ((nu - 1 - b) / G + 1) : 0;
  const int gq = G / S, gr = G % S;
  const int nt0 = (t.Nv[0] + 15) / 16;
  auto unit = [&](int tile, int slot, PItem& it) {
    it.tile = tile;
    it.slot = slot;
    it.cb = tile / nt0;
    it.ca = (tile - it.cb * nt0) * 16;
    it.nv = min(16, t.Nv[0] - it.ca);
  };
  auto issue = [&](const PItem& it) {
    if (t.skip_loads) return;
    fp::mbar_expect_tx(&tbar, 8u * U::TILE);
    fp::tma_load_tile(st, &in_map, it.ca, t.axis == 2 ? it.cb : 0, t.axis == 1 ? it.cb : 0,
                      shared_input ? 0 : it.slot, &tbar);
  };
  uint32_t mph = 0;
  bool failed = false;
  PItem cur, nxt;
  bool has_next = false;
  int inflight = -1;  // item whose tile load is issued and not yet waited for
  // one stage: the MMAs of all products, then a bounded wait for them; stage
  // 0 also issues the next tile's load (its operand has read the buffer)
  auto stage = [&](int s, int j) -> bool {
    um::fence_smem_async();
    um::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      um::fence_after_sync();
      const uint32_t a0 = um::saddr(Ahi), a1 = um::saddr(Alo);
      const int blk = F2 == 16 ? 0 : ((s == 0 || s == 3) ? 0 : 1);
      const uint32_t b0 = um::saddr(Bm + (2 * blk) * U::BBYTES), b1 = b0 + U::BBYTES;
      const uint32_t lboA = 256 * 16, lboB = 32 * 16;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int ks = 0; ks < U::KS; ++ks) {
          const uint32_t oa = h * 128 * 16 + ks * 2 * lboA, ob = ks * 2 * lboB;
          const uint64_t dAh = um::sdesc(a0 + oa, lboA, 128), dAl = um::sdesc(a1 + oa, lboA, 128);
          const uint64_t dBh = um::sdesc(b0 + ob, lboB, 128), dBl = um::sdesc(b1 + ob, lboB, 128);
          const uint32_t d = tmem + 32 * h;
          if (TF32) {
            um::mma_tf32(d, dAh, dBh, idd, ks > 0 ? 1u : 0u);
            um::mma_tf32(d, dAh, dBl, idd, 1u);
            um::mma_tf32(d, dAl, dBh, idd, 1u);
          } else {
            um::mma_bf16(d, dAh, dBh, idd, ks > 0 ? 1u : 0u);
            um::mma_bf16(d, dAh, dBl, idd, 1u);
            um::mma_bf16(d, dAl, dBh, idd, 1u);
          }
        }
      }
      um::commit(&mbar);
      if (s == 0 && has_next) {
        fp::fence_async_smem();
        issue(nxt);
      }
    }
    if (s == 0 && has_next) inflight = j + 1;
    const bool ok = um::bar_wait(&mbar, mph, kMmaWait);
    mph ^= 1;
    if (__syncthreads_or(!ok)) return false;
    um::fence_after_sync();
    return true;
  };

  if (n_items > 0) unit(b / S, b % S, cur);
  if (n_items > 0 && tid == 0) issue(cur);
  if (n_items > 0) inflight = 0;
  for (int j = 0; j < n_items && !failed; ++j) {
    // seeds of this thread's line (row (line, k1) of stage 2)
    float2 slo, shi, sst;
    {
      const int c0 = cur.ca + (ml < cur.nv ? ml : 0);
      const int row = t.a.Sd.b == 0 ? c0 : ((t.a.Sd.b < 0 || t.a.Sd.b == t.axis) ? 0 : cur.cb);
      const float2* sr = t.a.Sd.p + cur.slot * t.a.Sd.sstride + row * t.a.sd_w;
      slo = sr[mu];
      shi = sr[16 + mu];
      sst = sr[32];
    }
    bool late = false;
    if (tid == 0) fp::bulk_wait_read0();  // the previous result's store has read the operand area
    {
      uint32_t spins = 0;
      while (!fp::mbar_try_wait(&tbar, (uint32_t)(j & 1)))
        if (++spins > t.wait_limit) {
          late = true;
          break;
        }
    }
    if (__syncthreads_or(late)) {
      failed = true;
      break;
    }
    inflight = -1;
    has_next = j + 1 < n_items;
    if (has_next) {
      int slot = cur.slot + gr, tile = cur.tile + gq;
      if (slot >= S) {
        slot -= S;
        ++tile;
      }
      unit(tile, slot, nxt);
    }
    float2 v[16];
    // stage 1 operand: own row (line, t), K = m
    {
      const int tt = mu;
#pragma unroll
      for (int m = 0; m < 16; ++m) v[m] = tt < F2 ? st[fp::tswz(tt + F2 * m, ml)] : make_float2(0.f, 0.f);
      put_row<TF32>(Ahi, Alo, myrow, v);
    }
    if (!stage(0, j)) {
      failed = true;
      break;
    }
    // stage 1 -> 2: twiddle W_N^{t k1}, scatter into rows (line, k1), K = t
    row_load(trow, v);
    {
      const int tt = mu;
#pragma unroll
      for (int k1 = 0; k1 < 16; ++k1) {
        const float2 z = tt < F2 ? cmul(v[k1], tws[tt * 16 + k1]) : make_float2(0.f, 0.f);
        put_pair<TF32>(Ahi, Alo, rho(ml, k1), 256, tt, z);
      }
    }
    if (!stage(1, j)) {
      failed = true;
      break;
    }
    // stage 2 -> 3: X[k1 + 16 k2] times the phase factor, conjugated (stage 3
    // runs the forward W_F2 block), own row, K = k2
    row_load(trow, v);
    {
      constexpr int KP = F2 / 2;
      constexpr bool ODD = (F2 & 1) != 0;
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) {
        if (k2 >= F2) {
          v[k2] = make_float2(0.f, 0.f);
          continue;
        }
        float2 c;
        if (k2 < KP) {
          c = slo;
          if (k2 + 1 < KP || ODD) slo = cmul(slo, sst);
        } else if (ODD && k2 == KP) {
          c = (2 * mu < 16) ? slo : cmul(shi, cconj(sst));
        } else {
          c = shi;
          if (k2 + 1 < F2) shi = cmul(shi, sst);
        }
        v[k2] = cconj(cmul(c, v[k2]));
      }
      put_row<TF32>(Ahi, Alo, myrow, v);
    }
    if (!stage(2, j)) {
      failed = true;
      break;
    }
    // stage 3 -> 4: the accumulator holds conj(z); conj(z W_N^{-t k1}) =
    // conj(z) W_N^{t k1}, scattered into rows (line, t), K = k1
    row_load(trow, v);
    {
      const int k1 = mu;
#pragma unroll
      for (int tt = 0; tt < 16; ++tt) {
        const float2 z = tt < F2 ? cmul(v[tt], tws[tt * 16 + k1]) : make_float2(0.f, 0.f);
        put_pair<TF32>(Ahi, Alo, rho(ml, tt), 256, k1, z);
      }
    }
    if (!stage(3, j)) {
      failed = true;
      break;
    }
    // stage 4 result: row (line, t) holds conj(y[t + F2 m]); staged in the
    // operand area (the MMAs that read it are complete) for the TMA store
    row_load(trow, v);
    if (mu < F2) {
#pragma unroll
      for (int m = 0; m < 16; ++m) res[fp::tswz(mu + F2 * m, ml)] = cconj(v[m]);
    }
    fp::fence_async_smem();  // the writes above are read by the bulk store
    __syncthreads();
    if (tid == 0) {
      fp::tma_store_tile(&out_map, cur.ca, t.axis == 2 ? cur.cb : 0, t.axis == 1 ? cur.cb : 0, cur.slot, res);
      fp::bulk_commit();
    }
    cur = nxt;
  }
  if (failed && tid == 0) {
    atomicExch(t.err, 1);
    // a tile load still in flight lands before the shared memory is released
    if (inflight >= 0 && !t.skip_loads)
      for (uint32_t k = 0; k < t.wait_limit && !fp::mbar_try_wait(&tbar, (uint32_t)(inflight & 1)); ++k) {
      }
  }
  if (tid == 0) fp::bulk_wait0();
  um::fence_before_sync();
  __syncthreads();
  if (w == 0) um::tmem_dealloc(tmem, 64);
}

template <int F2, bool TF32>
bool launch_umma(const CUtensorMap& in, const CUtensorMap& out, const TArgs& t, const float2* tw, int shared_input,
                 int sm_count, cudaStream_t s) {
  using U = UCfg<F2, TF32>;
  static const bool ok = [] {
    // the largest shared-memory carveout, so that two CTAs fit on an SM
    const bool r = cudaFuncSetAttribute(umma_line_kernel<F2, TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)U::SMEM) == cudaSuccess &&
                   cudaFuncSetAttribute(umma_line_kernel<F2, TF32>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                        (int)cudaSharedmemCarveoutMaxShared) == cudaSuccess;
    cudaGetLastError();
    return r;
  }();
  if (!ok) return false;
  const long long tiles = (long long)((t.Nv[0] + 15) / 16) * t.Nv[t.axis == 1 ? 2 : 1];
  const long long units = tiles * t.n_vol;
  if (units == 0 || units >= (1LL << 31)) return false;
  static const int per_sm = [] {
    const int n = dis_ctas_per_sm(reinterpret_cast<const void*>(umma_line_kernel<F2, TF32>), kUT, U::SMEM);
    return n < 1 ? 1 : (n > 4 ? 4 : n);  // at most 4 x 64 tensor-memory columns per SM
  }();
  const long long cap = (long long)sm_count * per_sm;
  const unsigned grid = (unsigned)(units < cap ? units : cap);
  umma_line_kernel<F2, TF32><<<grid, kUT, U::SMEM, s>>>(in, out, t, tw, (int)tiles, shared_input);
  return true;
}

}  // namespace

// The transform line pass of lines of n points on the tensor cores (mode:
// DISORDER_PRECISION_BF16X3 or _TF32X3). False when no kernel exists for n.
bool dis_umma_line(int n, int mode, const CUtensorMap& in, const CUtensorMap& out, const TArgs& t, const float2* tw,
                   int shared_input, int sm_count, cudaStream_t s) {
  const bool tf = mode == DISORDER_PRECISION_TF32X3;
  switch (n) {
    case 256: return tf ? launch_umma<16, true>(in, out, t, tw, shared_input, sm_count, s)
                        : launch_umma<16, false>(in, out, t, tw, shared_input, sm_count, s);
    case 176: return tf ? launch_umma<11, true>(in, out, t, tw, shared_input, sm_count, s)
                        : launch_umma<11, false>(in, out, t, tw, shared_input, sm_count, s);
    default: return false;
  }
}
