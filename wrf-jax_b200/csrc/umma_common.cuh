// Device helpers shared by the tcgen05 kernels of the radiation surrogate:
// shared-memory matrix descriptors of the 128-byte swizzled K-major layout,
// bounded mbarrier waits, bulk copies, and the activation functions (one
// definition, so the unfused GEMM epilogues and the fused inference kernel
// round alike, in training and inference).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rrtmg {
namespace umma {

constexpr uint32_t kSbo = 1024;              // next 8-row group (8 rows x 128 B)
constexpr uint64_t kWaitNs = 2000000000ull;  // bounded mbarrier wait: 2 s

// tcgen05 instruction descriptor of a kind::f16 MMA with BF16 A and B (bits
// 7-9, 10-12 = 1), FP32 accumulate (bits 4-5 = 1), both operands K-major,
// N >> 3 at bit 17 and M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor of a K-major operand in the 128-byte
// swizzled layout: start address, leading-byte offset 16 (unused by this
// layout), stride-byte offset 1024 between 8-row groups (all in 16-byte
// units), descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1) << 16;
  d |= static_cast<uint64_t>((kSbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(2) << 61;
  return d;
}

// Byte offset of the 16-byte chunk kc (0..7) of row r in a 128-byte swizzled
// tile: rows are 128 B apart and the chunk index is XORed with r mod 8 (the
// hardware applies the same XOR to the addresses the descriptors produce).
__host__ __device__ __forceinline__ uint32_t swz(int r, int kc) {
  return static_cast<uint32_t>(r) * 128u + (static_cast<uint32_t>(kc ^ (r & 7)) << 4);
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t addr, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(addr), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the given phase parity of an mbarrier; gives up after limit_ns.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity, uint64_t limit_ns = kWaitNs) {
  const uint64_t t0 = global_ns();
  while (true) {
    if (mbar_try(addr, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// As mbar_wait, and also gives up as soon as *abort is set by another role.
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t addr, uint32_t parity, const volatile int *abort) {
  const uint64_t t0 = global_ns();
  while (true) {
    if (mbar_try(addr, parity)) return true;
    if (*abort) return false;
    if (global_ns() - t0 > kWaitNs) return false;
  }
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t addr) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(addr) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes) : "memory");
}

// One-dimensional bulk copy global -> shared memory of this CTA, completing
// on an mbarrier's transaction count; both addresses 16-byte aligned, size a
// multiple of 16.  No cluster multicast.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// Arrives on an mbarrier once every tcgen05 operation this thread issued
// before has completed.
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one kind::f16 MMA (K = 16).
__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's lane (row).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 8 consecutive 32-bit tensor-memory columns of this thread's lane: load, store.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
               "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// GELU in the tanh form of Hendrycks & Gimpel (2016), 0.5 z (1 + tanh(u)),
// u = sqrt(2/pi) (z + 0.044715 z^3), with the hardware tanh (one MUFU
// operation), and its derivative 0.5 (1 + t) + 0.5 z (1 - t^2) du/dz.
__device__ __forceinline__ float gelu(float z) {
  const float h = 0.5f * z;
  const float u = z * fmaf(0.0356774081f, z * z, 0.7978845608f);
  return fmaf(h, tanh_approx(u), h);
}

__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float t = tanh_approx(z * fmaf(0.0356774081f, z2, 0.7978845608f));
  const float du = fmaf(0.1070322243f, z2, 0.7978845608f);
  return fmaf(0.5f, t, 0.5f) + (0.5f * z) * fmaf(-t, t, 1.0f) * du;
}

}  // namespace umma
}  // namespace rrtmg
