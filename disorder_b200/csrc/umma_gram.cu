// Coil-compression Gram matrix on the tensor cores (mixed precision).
//
// compressCoils (Methods/compressCoils.m:78-88) forms the C x C Hermitian
// matrix P(c, d) = sum_v a_c(v) conj(S_d(v)) with a = S / (sum_c |S_c|^2 + reg):
// one contraction over every voxel of the volume. As a real GEMM over
// K = (voxel, re/im):
//   A row 2c   = [a_re,  a_im] per voxel,   A row 2c+1 = [a_im, -a_re],
//   B row d    = [S_re,  S_im] per voxel,
// so D(2c, d) = Re P(c, d) and D(2c+1, d) = Im P(c, d); M = 128 rows (2C used),
// N = C rounded up to 16. Each CTA walks chunks of voxels: the threads stage
// the chunk's coil values, scale them, split every operand into two
// tensor-core parts (BF16x3: bf16 hi + bf16 lo; 3xTF32: tf32 hi + tf32 lo) and
// write them K-major; one thread issues hi*hi + hi*lo + lo*hi into the FP32
// accumulator in tensor memory. Every kFlush chunks the accumulator is read
// into per-thread FP64 sums (row = thread) and restarted, so the FP32
// accumulation spans at most kFlush * chunk voxels. The per-CTA FP64 partials
// have the layout of the CUDA-core Gram's, and the host adds them up.
//
// Waits on the MMA completion are bounded; a wait that runs out sets the
// error word and the CTA stops, after a second bounded wait, freeing its
// tensor memory.
#include "internal.h"
#include "umma.cuh"

namespace {

constexpr int kGT = 128;    // threads: thread t owns accumulator row t
constexpr int kFlush = 8;   // chunks per FP32 accumulation span
constexpr uint32_t kWait = 1u << 20;

template <bool TF32>
struct GramCfg {
  static constexpr int KV = TF32 ? 32 : 64;          // voxels per chunk
  static constexpr int K = 2 * KV;                   // real K per chunk
  static constexpr int ES = TF32 ? 4 : 2;            // operand element size
  static constexpr int E = 16 / ES;                  // elements per 16-byte chunk
  static constexpr int KSTEP = TF32 ? 8 : 16;        // K per MMA
  static constexpr size_t A_BYTES = (size_t)128 * K * ES;
  static constexpr size_t B_BYTES = (size_t)64 * K * ES;  // N <= 64
  static constexpr size_t S_BYTES = (size_t)64 * KV * sizeof(float2);
  static constexpr size_t SMEM = 2 * A_BYTES + 2 * B_BYTES + S_BYTES + KV * sizeof(float) + 1024;
};

// byte offset of element (r, k) of an R-row K-major operand
template <bool TF32>
DIS_D uint32_t op_off(int r, int k, int R) {
  using G = GramCfg<TF32>;
  return (uint32_t)((k / G::E) * (R * 16) + r * 16 + (k % G::E) * G::ES);
}

template <bool TF32>
__global__ void __launch_bounds__(kGT, 1)
    gram_umma_kernel(const float2* __restrict__ S, int C, long long V, float reg, double* __restrict__ part,
                     int* err) {
  using G = GramCfg<TF32>;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* Ahi = sm;
  unsigned char* Alo = Ahi + G::A_BYTES;
  unsigned char* Bhi = Alo + G::A_BYTES;
  unsigned char* Blo = Bhi + G::B_BYTES;
  float2* sS = reinterpret_cast<float2*>(Blo + G::B_BYTES);  // [C][KV]
  float* sinv = reinterpret_cast<float*>(sS + 64 * G::KV);
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  __shared__ int stop;
  const int tid = threadIdx.x;
  const int NB = C <= 16 ? 16 : (C <= 32 ? 32 : (C <= 48 ? 48 : 64));
  const uint32_t ncols = NB <= 32 ? 32 : 64;
  // zero the operands once: rows >= 2C of A and >= C of B stay zero
  for (size_t e = tid; e < (2 * G::A_BYTES + 2 * G::B_BYTES) / 16; e += kGT)
    reinterpret_cast<uint4*>(sm)[e] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    um::bar_init(&bar, 1);
    stop = 0;
  }
  if (tid < 32) {
    um::tmem_alloc(&tbase, ncols);
    um::tmem_relinquish();
  }
  um::fence_before_sync();
  __syncthreads();
  um::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t id = um::idesc(TF32 ? um::kTF32 : um::kBF16, 128, NB);
  double acc[64];
#pragma unroll
  for (int n = 0; n < 64; ++n) acc[n] = 0.0;
  uint32_t phase = 0;
  int since = 0;  // chunks accumulated in tensor memory since the last flush
  const long long nchunks = (V + G::KV - 1) / G::KV;

  auto flush = [&]() {
    um::fence_after_sync();
    const uint32_t lane_addr = tmem + ((uint32_t)(tid & ~31) << 16);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q * 16 < NB) {
        float v[16];
        um::tld16(lane_addr + q * 16, v);
        um::tld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[q * 16 + i] += (double)v[i];
      }
    }
    um::fence_before_sync();
  };

  for (long long ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const long long v0 = ch * G::KV;
    // stage the chunk's coil values [C][KV] (coalesced along voxels)
    for (int e = tid; e < C * G::KV; e += kGT) {
      const int c = e / G::KV, j = e % G::KV;
      const long long v = v0 + j;
      sS[e] = v < V ? S[(long long)c * V + v] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    if (tid < G::KV) {
      float n = 0.f;
      for (int c = 0; c < C; ++c) {
        const float2 a = sS[c * G::KV + tid];
        n = fmaf(a.x, a.x, fmaf(a.y, a.y, n));
      }
      sinv[tid] = 1.0f / (n + reg);
    }
    __syncthreads();
    // operands: the (re, im) pair of voxel j sits at K columns 2j, 2j+1
    for (int e = tid; e < C * G::KV; e += kGT) {
      const int c = e / G::KV, j = e % G::KV;
      const float2 s = sS[e];
      const float2 a = cscale(s, sinv[j]);
      if (TF32) {
        float h0, l0, h1, l1;
        auto put = [&](unsigned char* hb, unsigned char* lb, int r, int R, float x, float y) {
          um::split_tf32(x, h0, l0);
          um::split_tf32(y, h1, l1);
          const uint32_t o = op_off<TF32>(r, 2 * j, R);
          *reinterpret_cast<float2*>(hb + o) = make_float2(h0, h1);
          *reinterpret_cast<float2*>(lb + o) = make_float2(l0, l1);
        };
        put(Ahi, Alo, 2 * c, 128, a.x, a.y);
        put(Ahi, Alo, 2 * c + 1, 128, a.y, -a.x);
        put(Bhi, Blo, c, NB, s.x, s.y);
      } else {
        uint32_t h, l;
        auto put = [&](unsigned char* hb, unsigned char* lb, int r, int R, float x, float y) {
          um::split_bf16x2(x, y, h, l);
          const uint32_t o = op_off<TF32>(r, 2 * j, R);
          *reinterpret_cast<uint32_t*>(hb + o) = h;
          *reinterpret_cast<uint32_t*>(lb + o) = l;
        };
        put(Ahi, Alo, 2 * c, 128, a.x, a.y);
        put(Ahi, Alo, 2 * c + 1, 128, a.y, -a.x);
        put(Bhi, Blo, c, NB, s.x, s.y);
      }
    }
    um::fence_smem_async();
    __syncthreads();
    if (tid == 0) {
      um::fence_after_sync();
      const uint32_t a0 = um::saddr(Ahi), a1 = um::saddr(Alo), b0 = um::saddr(Bhi), b1 = um::saddr(Blo);
      const uint32_t lboA = 128 * 16, lboB = NB * 16;
#pragma unroll 1
      for (int ks = 0; ks < G::K / G::KSTEP; ++ks) {
        const uint32_t oa = ks * 2 * lboA, ob = ks * 2 * lboB;
        const uint64_t dAh = um::sdesc(a0 + oa, lboA, 128), dAl = um::sdesc(a1 + oa, lboA, 128);
        const uint64_t dBh = um::sdesc(b0 + ob, lboB, 128), dBl = um::sdesc(b1 + ob, lboB, 128);
        const uint32_t first = (since == 0 && ks == 0) ? 0u : 1u;
        if (TF32) {
          um::mma_tf32(tmem, dAh, dBh, id, first);
          um::mma_tf32(tmem, dAh, dBl, id, 1);
          um::mma_tf32(tmem, dAl, dBh, id, 1);
        } else {
          um::mma_bf16(tmem, dAh, dBh, id, first);
          um::mma_bf16(tmem, dAh, dBl, id, 1);
          um::mma_bf16(tmem, dAl, dBh, id, 1);
        }
      }
      um::commit(&bar);
    }
    // the MMAs have read the operands (and written the accumulator)
    if (!um::bar_wait(&bar, phase, kWait)) atomicExch(&stop, 1);
    phase ^= 1;
    __syncthreads();
    if (stop) break;
    if (++since == kFlush) {
      flush();
      since = 0;
    }
  }
  if (!stop && since > 0) flush();
  if (stop) {
    if (tid == 0) atomicExch(err, 1);
    um::bar_wait(&bar, phase, kWait);  // an MMA group may still be in flight
  }
  __syncthreads();
  if (tid < 32) um::tmem_dealloc(tmem, ncols);
  if (stop) return;
  // row tid = 2c + o: o = 0 the real parts of P(c, :), o = 1 the imaginary parts
  if (tid < 2 * C) {
    const int c = tid >> 1, o = tid & 1;
    double* dst = part + (size_t)blockIdx.x * C * C * 2;
#pragma unroll
    for (int d = 0; d < 64; ++d)
      if (d < C) dst[((size_t)c * C + d) * 2 + o] = acc[d];
  }
}

}  // namespace

// Partial Gram matrices of compressCoils on the tensor cores: part[b][c*C+d]
// (re, im) for b < grid. mode: DISORDER_PRECISION_BF16X3 or _TF32X3.
int dis_gram_umma(disorder_ctx_s* ctx, const float2* S, int C, long long V, float reg, double* part, int grid,
                  int mode) {
  if (C < 1 || C > 64) return dis_set_error(ctx, DISORDER_BAD_ARG, "gram: 1 <= C <= 64");
  const bool tf32 = mode == DISORDER_PRECISION_TF32X3;
  const size_t smem = tf32 ? GramCfg<true>::SMEM : GramCfg<false>::SMEM;
  if (tf32) {
    DIS_CUDA_TRY(cudaFuncSetAttribute(gram_umma_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gram_umma_kernel<true><<<grid, kGT, smem, ctx->stream>>>(S, C, V, reg, part, ctx->d_err);
  } else {
    DIS_CUDA_TRY(cudaFuncSetAttribute(gram_umma_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    gram_umma_kernel<false><<<grid, kGT, smem, ctx->stream>>>(S, C, V, reg, part, ctx->d_err);
  }
  dis_count(ctx);
  DIS_CUDA_TRY(cudaGetLastError());
  return DISORDER_OK;
}
