// Strided line passes with TMA tile copies (sm_100a).
//
// The strided passes (lines along dim 2 or 3 of a volume, 16 lines adjacent
// along dim 1 per tile) of the sinc rigid transform and the weighted dim-2
// pass of the normal operator spend most of their load/store issue slots on
// per-element copies when the copies go through the threads (8-byte cp.async
// in, 16-byte stores out). Here one thread moves a whole tile each way with
// cp.async.bulk.tensor: a 4-D tensor map {N0, N1, N2, volume} in memory
// order with box {16, N, 1, 1} (pass along dim 2) or {16, 1, N, 1} (along
// dim 3) and the 128-byte swizzle, so the tile lands in
// shared memory as 128-byte rows (one row per position along the pass axis)
// whose 16-byte chunks are XOR-permuted by the row index mod 8 - the layout
// the layout-A reads need to avoid bank conflicts. Loads complete on an
// mbarrier per stage buffer (double buffered); the result tile is written
// back in place and stored by the same thread with one bulk tensor store.
//
// No load here uses cluster multicast, and the tensor maps only cover this
// GPU's own buffers.
//
// Waits on the mbarriers are bounded: a wait that runs out sets the
// context's device error word (TArgs::err) and the CTA stops after its
// stores in flight complete; disorder_synchronize reports it as
// DISORDER_TIMEOUT.
#pragma once
#include <cuda.h>

#include "pipepass.cuh"

namespace fp {

DIS_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

DIS_D void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
DIS_D void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
DIS_D bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
DIS_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// tile load of the map's box at {x, y, z, w} into dst, completing on bar
DIS_D void tma_load_tile(void* dst, const CUtensorMap* map, int x, int y, int z, int w, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}
DIS_D void tma_store_tile(const CUtensorMap* map, int x, int y, int z, int w, const void* src) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(src))
               : "memory");
}
DIS_D void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
DIS_D void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
DIS_D void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// element (p, l) of a tile copied with the 128-byte swizzle (rows of 16
// complex64 elements, buffer 1024-byte aligned)
DIS_D int tswz(int p, int l) { return p * 16 + ((((l >> 1) ^ (p & 7)) << 1) | (l & 1)); }

template <int F1, int F2>
struct TPipe {
  using LN = ff::Line<F1, F2>;
  static constexpr int N = LN::N, TL = LN::TL, LPB = kThreads / TL;
  static_assert(LPB == 16, "TMA tiles are 16 lines (128-byte rows)");
  static constexpr int TILE = N * LPB, EXT = LPB * LN::EXSZ;
  static constexpr int SBB = ((8 * (TILE > EXT ? TILE : EXT)) + 1023) & ~1023;  // stage buffer bytes
  static constexpr int TWB = ((8 * LN::TWS) + 15) & ~15;
  static constexpr size_t SMEM = 1024 + 2 * (size_t)SBB + TWB;  // + alignment slack
  static constexpr uint32_t BOX_BYTES = 8u * TILE;
};

// KIND 0: transform pass (coefficient from the line's phase seeds, a.Sd);
// KIND 1: normal-operator weighting (coefficient = sample weight, volumes are
// the per-coil intermediates, unit = (tile, slot) walking its C coils); with
// t.y set it also writes the tile's samples of the forward DFT (what encode
// would produce for the same input) before weighting them;
// KIND 2: encode gather (DFT along dim 2, then the segment's samples of the
// tile's ky rows are read out of the tile into y; no store);
// KIND 3: decode scatter (the tile is built from the weighted samples, then
// the inverse DFT along dim 2 is stored; no load). Kinds 1-3 share the unit
// walk over (tile, slot) and its C coils.
// Geometry: volumes of Nv = {N0, N1, N2} with the pass along `axis` (1 or 2);
// tile = 16 lines adjacent along N0 at one position of the other axis.
struct TArgs {
  int Nv[3];
  int axis;
  int n_vol;       // volumes (KIND 0: slots; KIND 1: slots * C)
  int n_slots, C;  // KIND 1
  const int* slot_seg;
  const float* wmap;  // KIND 1: [seg][N0][N_pass]
  LinePassArgs a;     // KIND 0: seeds
  int* err;           // device error word (set to 1 when a wait runs out)
  // bound of every tile wait, in try_wait rounds (each suspends for a short
  // hardware-defined time; the default is of the order of a second)
  unsigned wait_limit = 1u << 20;
  // failure-path testing (disorder_ctx_inject_fault): issue no tile load, so
  // the first wait of every CTA runs out with nothing in flight
  int skip_loads = 0;
  // KIND 2 / 3: per-segment CSR of the samples by ky row, sample rows and
  // the sample array y[ld*(n3 + n3off) + ld*N3y*c + i]
  const int* rowptr;
  const int* perm;
  const int* kyv;
  const int* kzv;
  float2* y;
  const float2* ymeas;  // KIND 2: subtracted when non-null
  long long ld;
  int n3off, N3y;
  float scale;          // KIND 2
  const float* We;      // KIND 3: per-sample weights or null
  const float* Mb;      // KIND 3: readout weights or null
};

template <int F1, int F2, int KIND>
__global__ void __launch_bounds__(kThreads, 3)
    tma_kernel(const __grid_constant__ CUtensorMap in_map, const __grid_constant__ CUtensorMap out_map, TArgs t,
               const float2* __restrict__ twg, int n_tiles, int shared_input) {
  using P = TPipe<F1, F2>;
  using LN = typename P::LN;
  constexpr int TL = P::TL;
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ uint64_t mbar[2];
  // 1024-byte aligned stage buffers, then the twiddles
  const uint32_t base_s = smem_u32(smraw);
  unsigned char* al = smraw + (((base_s + 1023u) & ~1023u) - base_s);
  float2* stg0 = reinterpret_cast<float2*>(al);
  float2* stg1 = reinterpret_cast<float2*>(al + P::SBB);
  float2* tw = reinterpret_cast<float2*>(al + 2 * P::SBB);
  const int tid = threadIdx.x, lt = tid % TL, li = tid / TL;
  ff::load_tw<F1, F2>(tw, twg, tid, kThreads);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_async_smem();
  }
  __syncthreads();
  const int G = gridDim.x, b = blockIdx.x;
  constexpr bool LOAD = KIND != 3, STORE = KIND != 2;
  const int S = KIND >= 1 ? t.n_slots : t.n_vol, C = KIND >= 1 ? t.C : 1;
  const int nu = n_tiles * S;  // units: tile u / S, slot u % S
  const int n_items = b < nu ? ((nu - 1 - b) / G + 1) * C : 0;
  if (n_items == 0) return;
  const int gq = G / S, gr = G % S;
  const int nt0 = (t.Nv[0] + 15) / 16;
  auto unit = [&](int tile, int slot, PItem& it) {
    it.tile = tile;
    it.slot = slot;
    it.cb = tile / nt0;
    it.ca = (tile - it.cb * nt0) * 16;
    it.nv = min(16, t.Nv[0] - it.ca);
  };
  auto issue = [&](const PItem& it, int c, float2* st, uint64_t* bar) {
    if (t.skip_loads) return;
    mbar_expect_tx(bar, P::BOX_BYTES);
    const int w = KIND >= 1 ? it.slot * C + c : (shared_input ? 0 : it.slot);
    tma_load_tile(st, &in_map, it.ca, t.axis == 2 ? it.cb : 0, t.axis == 1 ? it.cb : 0, w, bar);
  };
  // KIND 1 (with samples) / 2: the tile's samples of the forward DFT, warp
  // by warp from registers. A warp holds two lines (16 threads each); the
  // sample at (line, kz) is X[kz / F1] of lane 16 (line & 1) + kz % F1, so
  // each lane takes one of the warp's samples (the segment's CSR over the two
  // ky rows) and reads it with shuffles; no CTA barrier, no copy of the tile.
  auto warp_samples = [&](const PItem& it, int c, float2 (&Xr)[F2], const float2* ymeas, float scale) {
    if (lt >= F1) {
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) Xr[k2] = make_float2(0.f, 0.f);
    }
    const int lane = tid & 31, wl0 = (tid >> 5) * 2;
    const int* rp = t.rowptr + (long long)t.slot_seg[it.slot] * (t.Nv[0] + 1);
    const int qa = rp[it.ca + min(wl0, it.nv)], qe = rp[it.ca + min(wl0 + 2, it.nv)];
    const long long ob = t.ld * (it.cb + t.n3off) + t.ld * t.N3y * c;
    for (int qb = qa; qb < qe; qb += 32) {
      const int q = qb + lane;
      const bool have = q < qe;
      int i = 0, src = 0, kk = -1;
      if (have) {
        i = t.perm[q];
        const int kz = t.kzv[i], row = t.kyv[i] - it.ca - wl0;
        if (DIS_DEBUG_INDEX(kz, t.Nv[t.axis], t.err, DIS_SITE_TMA_SAMPLES) &&
            DIS_DEBUG_INDEX(row, 2, t.err, DIS_SITE_TMA_SAMPLES)) {
          src = 16 * row + kz % F1;
          kk = kz / F1;
        }
      }
      float2 val = make_float2(0.f, 0.f);
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) {
        const float vx = __shfl_sync(0xffffffffu, Xr[k2].x, src);
        const float vy = __shfl_sync(0xffffffffu, Xr[k2].y, src);
        if (kk == k2) val = make_float2(vx, vy);
      }
      if (have) {
        float2 o = cscale(val, scale);
        if (ymeas) o = csub(o, ymeas[ob + i]);
        t.y[ob + i] = o;
      }
    }
  };
  PItem cur;
  unit(b / S, b % S, cur);
  int cc = 0;
  if (LOAD && tid == 0) issue(cur, 0, stg0, &mbar[0]);
  for (int j = 0; j < n_items; ++j) {
    float2* st = (j & 1) ? stg1 : stg0;
    const bool valid = li < cur.nv;
    // coefficient sources of this line (loaded while the tile lands)
    float2 slo, shi, sst;
    const float* wm = nullptr;
    if (KIND == 0 && lt < F1) {
      const int c0 = cur.ca + (valid ? li : 0);
      const int row = t.a.Sd.b == 0 ? c0 : ((t.a.Sd.b < 0 || t.a.Sd.b == t.axis) ? 0 : cur.cb);
      const float2* sr = t.a.Sd.p + cur.slot * t.a.Sd.sstride + row * t.a.sd_w;
      slo = sr[lt];
      shi = sr[F1 + lt];
      sst = sr[2 * F1];
    }
    if (KIND == 1)
      wm = t.wmap + ((long long)t.slot_seg[cur.slot] * t.Nv[0] + cur.ca + (valid ? li : 0)) * t.Nv[t.axis];
    // bounded wait for the tile (each try_wait suspends for a short
    // hardware-defined time; the default bound is of the order of a second)
    bool late = false;
    if (LOAD) {
      uint32_t spins = 0;
      while (!mbar_try_wait(&mbar[j & 1], (uint32_t)((j >> 1) & 1))) {
        if (++spins > t.wait_limit) {
          late = true;
          break;
        }
      }
    }
    // every thread is past item j-1 (its reads of the other buffer included)
    if (__syncthreads_or(late)) {
      if (tid == 0) {
        atomicExch(t.err, 1);
        // the only load that can be in flight is item j's (item j+1's is
        // issued after this wait): give it another bounded wait to land
        // before the CTA's shared memory is released, then drain the stores
        if (LOAD && !t.skip_loads)
          for (uint32_t k = 0; k < t.wait_limit && !mbar_try_wait(&mbar[j & 1], (uint32_t)((j >> 1) & 1)); ++k) {
          }
        bulk_wait0();
      }
      return;
    }
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
        unit(tile, slot, nxt);
      }
      if (LOAD && tid == 0) {
        if (STORE) bulk_wait_read0();  // item j-1's store has read the other buffer
        fence_async_smem();
        issue(nxt, cn, (j & 1) ? stg0 : stg1, &mbar[(j + 1) & 1]);
      }
    }
    float2 v[F1], X[F2];
    float2* myex = st + li * LN::EXSZ;
    if (KIND >= 2) {
      // this unit's sample range: segment rows ky in [ca, ca + nv)
      const int* rp = t.rowptr + (long long)t.slot_seg[cur.slot] * (t.Nv[0] + 1);
      const int s0 = rp[cur.ca], s1 = rp[cur.ca + cur.nv];
      const long long ob = t.ld * (cur.cb + t.n3off) + t.ld * t.N3y * cc;
      if (KIND == 2) {
#pragma unroll
        for (int m = 0; m < F1; ++m) v[m] = (lt < F2) ? st[tswz(lt + F2 * m, li)] : make_float2(0.f, 0.f);
        __syncthreads();  // the tile becomes the exchange area
        LN::fwd(v, X, lt, myex, tw);
        warp_samples(cur, cc, X, t.ymeas, t.scale);
        cur = nxt;
        cc = cn;
        continue;
      }
      // KIND 3: the tile from the weighted samples (buffer free once every
      // earlier store has read it)
      if (tid == 0) bulk_wait_read0();
      __syncthreads();
      for (int e = tid; e < P::TILE / 2; e += kThreads)
        reinterpret_cast<float4*>(st)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
      __syncthreads();
      const float mb = t.Mb ? t.Mb[cur.cb + t.n3off] : 1.f;
      for (int q = s0 + tid; q < s1; q += kThreads) {
        const int i = t.perm[q];
        const float w = t.We ? mb * t.We[i] : mb;
        const float2 val = cscale(t.y[ob + i], w);
        if (!DIS_DEBUG_INDEX(t.kzv[i], t.Nv[t.axis], t.err, DIS_SITE_TMA_SAMPLES) ||
            !DIS_DEBUG_INDEX(t.kyv[i] - cur.ca, cur.nv, t.err, DIS_SITE_TMA_SAMPLES))
          continue;
        float2* d = &st[tswz(t.kzv[i], t.kyv[i] - cur.ca)];
        atomicAdd(&d->x, val.x);
        atomicAdd(&d->y, val.y);
      }
      __syncthreads();
#pragma unroll
      for (int k2 = 0; k2 < F2; ++k2) X[k2] = lt < F1 ? st[tswz(lt + F1 * k2, li)] : make_float2(0.f, 0.f);
      __syncthreads();  // the tile becomes the exchange area
      LN::inv(X, v, lt, myex, tw);
    } else {
#pragma unroll
    for (int m = 0; m < F1; ++m) v[m] = (lt < F2) ? st[tswz(lt + F2 * m, li)] : make_float2(0.f, 0.f);
    __syncthreads();  // the tile becomes the exchange area
    LN::fwd(v, X, lt, myex, tw);
    // the segment's samples of this tile, as encode's gather writes them
    if (KIND == 1 && t.y) warp_samples(cur, cc, X, nullptr, t.scale);
    if (lt < F1) {
      if (KIND == 0) {
        constexpr int KP = F2 / 2;
        constexpr bool ODD = (F2 & 1) != 0;
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
      } else {
#pragma unroll
        for (int k2 = 0; k2 < F2; ++k2) X[k2] = cscale(X[k2], wm[lt + F1 * k2]);
      }
    }
    LN::inv(X, v, lt, myex, tw);
    }
    __syncthreads();  // every line's exchange is done
    if (lt < F2) {
#pragma unroll
      for (int m = 0; m < F1; ++m) st[tswz(lt + F2 * m, li)] = v[m];
    }
    fence_async_smem();  // the writes above are read by the bulk store
    __syncthreads();
    if (tid == 0) {
      const int w = KIND >= 1 ? cur.slot * C + cc : cur.slot;
      tma_store_tile(&out_map, cur.ca, t.axis == 2 ? cur.cb : 0, t.axis == 1 ? cur.cb : 0, w, st);
      bulk_commit();
    }
    cur = nxt;
    cc = cn;
  }
  if (STORE && tid == 0) bulk_wait0();
}

// Host side (tmamap.cu): the tensor map of n_vol volumes N0 x N1 x N2
// (complex64, volume stride vol_stride elements) for a pass along `axis`
// (1 or 2): dims {N0, N1, N2, n_vol} in memory order, box 16 x N[axis].
// False when the layout breaks a TMA rule (alignment, strides).
bool dis_tmap_volumes(CUtensorMap* m, const void* base, const int* N, int axis, long long vol_stride, int n_vol);

template <int F1, int F2>
struct TmaLaunch {
  using P = TPipe<F1, F2>;
  struct Occ {
    int per_sm[4] = {0, 0, 0, 0}, sms = 0;
  };
  template <int KIND>
  static void prep(Occ& o) {
    cudaFuncSetAttribute(tma_kernel<F1, F2, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P::SMEM);
    // the largest carveout, so the persistent grid's CTAs per SM are all resident
    cudaFuncSetAttribute(tma_kernel<F1, F2, KIND>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.per_sm[KIND], tma_kernel<F1, F2, KIND>, kThreads, P::SMEM);
  }
  static Occ init() {
    Occ o;
    prep<0>(o);
    prep<1>(o);
    prep<2>(o);
    prep<3>(o);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev);
    return o;
  }
  static bool launch(int kind, const CUtensorMap& in, const CUtensorMap& out, const TArgs& t, const float2* tw,
                     int shared_input, cudaStream_t s) {
    static const Occ occ = init();
    if (occ.per_sm[kind] <= 0 || occ.sms <= 0) return false;
    const long long tiles = (long long)((t.Nv[0] + 15) / 16) * t.Nv[t.axis == 1 ? 2 : 1];
    const int S = kind >= 1 ? t.n_slots : t.n_vol, C = kind >= 1 ? t.C : 1;
    const long long units = tiles * S;
    if (units == 0 || units * C >= (1LL << 31)) return false;
    const long long cap = (long long)occ.sms * occ.per_sm[kind];
    const unsigned grid = (unsigned)(units < cap ? units : cap);
    switch (kind) {
      case 0: tma_kernel<F1, F2, 0><<<grid, kThreads, P::SMEM, s>>>(in, out, t, tw, (int)tiles, shared_input); break;
      case 1: tma_kernel<F1, F2, 1><<<grid, kThreads, P::SMEM, s>>>(in, out, t, tw, (int)tiles, shared_input); break;
      case 2: tma_kernel<F1, F2, 2><<<grid, kThreads, P::SMEM, s>>>(in, out, t, tw, (int)tiles, shared_input); break;
      default: tma_kernel<F1, F2, 3><<<grid, kThreads, P::SMEM, s>>>(in, out, t, tw, (int)tiles, shared_input); break;
    }
    return true;
  }
};

}  // namespace fp

#define DIS_TMA_INSTANTIATE(F1, F2) template struct fp::TmaLaunch<F1, F2>;
