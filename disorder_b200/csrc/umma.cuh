// 5th-generation tensor-core primitives (tcgen05, sm_100a) for the
// mixed-precision contractions: tensor-memory allocation, shared-memory
// matrix descriptors, the MMA itself, its completion on an mbarrier, and
// tensor-memory loads into registers.
//
// Operand layout used throughout (K-major, no swizzle): an R-row x K-column
// operand (R = M rows of A or N rows of B) is stored as K/E chunks of E
// elements (16 bytes: 8 bf16 or 4 fp32), chunk-major; inside a chunk the R
// rows are consecutive 16-byte rows. Element (r, k) is at byte
//   (k / E) * (R * 16) + r * 16 + (k % E) * sizeof(elem).
// Eight consecutive rows of one chunk are one 128-byte core matrix, so the
// descriptor's stride offset (between 8-row groups) is 128 bytes and its
// leading offset (between the two K chunks of one bf16 MMA, K = 16) is
// R * 16 bytes.
//
// Accumulators: for cta_group::1 and M = 128, row m of D is tensor-memory
// lane m and column n is tensor-memory column (base + n), 32 bits each;
// warp w of the CTA reads lanes 32w..32w+31 with tcgen05.ld.
#pragma once
#include <cstdint>

#include "common.cuh"

namespace um {

DIS_D uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---- mbarriers (single arrival: the tcgen05.commit of the issuing thread)
DIS_D void bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(bar)), "r"(count) : "memory");
}
DIS_D bool bar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false when `limit` rounds of try_wait (each suspends for a
// short hardware-defined time) pass without the phase completing
DIS_D bool bar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t k = 0; k < limit; ++k)
    if (bar_try_wait(bar, parity)) return true;
  return false;
}
// generic-proxy shared-memory writes made visible to the tensor core
DIS_D void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ---- tensor memory
// whole warp: allocate ncols columns (a power of two >= 32), the address is
// written to *dst in shared memory
DIS_D void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(dst)), "r"(ncols)
               : "memory");
}
DIS_D void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory"); }
DIS_D void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
DIS_D void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
DIS_D void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// ---- descriptors
// shared-memory matrix descriptor: K-major, no swizzle, sm_100 version bits
DIS_D uint64_t sdesc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((start >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// instruction descriptor of kind::f16 (fmt 1: BF16 A and B) or kind::tf32
// (fmt 2): FP32 accumulator, K-major A and B, M x N
constexpr uint32_t idesc(uint32_t fmt, int M, int N) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
constexpr uint32_t kBF16 = 1, kTF32 = 2;

// ---- MMA (issued by one thread), accumulate when acc != 0
DIS_D void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc)
      : "memory");
}
DIS_D void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc)
      : "memory");
}
// the mbarrier receives one arrival when every MMA this thread issued so far
// has completed
DIS_D void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(saddr(bar))
               : "memory");
}

// ---- tensor memory -> registers: 32 lanes x 16 consecutive columns
DIS_D void tld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
DIS_D void tld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// ---- operand splitting for the three-product (x3) schemes
// BF16x3: v = hi + lo with hi = bf16(v), lo = bf16(v - hi); the products
// hi*hi + hi*lo + lo*hi keep about 16 significant bits of each operand.
DIS_D void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo) {
  uint32_t h;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;\n" : "=r"(h) : "f"(b), "f"(a));  // low half = a
  const float ah = __uint_as_float(h << 16), bh = __uint_as_float(h & 0xFFFF0000u);
  uint32_t l;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;\n" : "=r"(l) : "f"(b - bh), "f"(a - ah));
  hi = h;
  lo = l;
}
// 3xTF32: hi = v rounded to TF32 (10 explicit mantissa bits), lo = v - hi
// (read by the tensor core as TF32 too)
DIS_D void split_tf32(float v, float& hi, float& lo) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(h) : "f"(v));
  hi = __uint_as_float(h);
  lo = v - hi;
}

}  // namespace um
