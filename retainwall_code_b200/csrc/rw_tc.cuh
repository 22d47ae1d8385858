// Fifth-generation tensor core (tcgen05) building blocks for sm_100a: shared-memory
// matrix descriptors, the BF16 x BF16 -> FP32 instruction descriptor, tensor-memory
// (TMEM) allocation, MMA issue and completion through an mbarrier, TMEM loads, and the
// fences that order them against ordinary thread code.
//
// Operand layout used everywhere in this project: K-major, no swizzle (read transposed as
// MN-major by the weight-gradient products, see sdesc_mn).  A tile of R rows
// (M or N) by K columns of 16-bit elements is stored as 8-row x 16-byte core matrices;
// element (r, k) lives at byte
//     (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,   SBO = (K / 8) * 128,
// so the core matrices adjacent in K are 128 bytes apart (the descriptor's leading byte
// offset) and the 8-row groups SBO bytes apart (its stride byte offset).  One MMA
// instruction consumes K = 16, i.e. two core matrices along K; the next K step starts
// 256 bytes further.
#pragma once
#include <stdint.h>

namespace rw {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in a K-major, no-swizzle tile with K columns.
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (K-major, no swizzle): start address, leading byte
// offset (K direction), stride byte offset (8-row groups), descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: D FP32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// The same with A and B both MN-major (bits 15 and 16: the operands are read transposed).
__host__ __device__ constexpr uint32_t idesc_bf16_mn(int M, int N) {
  return idesc_bf16(M, N) | (1u << 15) | (1u << 16);
}

// A K-major, no-swizzle tile of 128 rows by Kc columns (the layout above) read as an
// MN-major operand whose MN index is the tile's column and whose K index is its row:
// the 8-row x 16-byte core matrices are then 8 K-rows of 8 MN elements, the core
// matrices adjacent in MN are 128 bytes apart (stride byte offset) and the groups of 8
// K-rows (Kc / 8) * 128 bytes apart (leading byte offset).  One MMA (K = 16) consumes
// two such groups; the next one starts Kc * 32 bytes further.
__device__ __forceinline__ uint64_t sdesc_mn(uint32_t saddr, int Kc) {
  return sdesc(saddr, (uint32_t)Kc * 16u, 128u);
}

// ---- mbarrier ------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase with the given parity to complete; gives up after max_iter polls
// (each try_wait itself suspends for a bounded time) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int max_iter = 1 << 20) {
  for (int it = 0; it < max_iter; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// ---- tensor memory -----------------------------------------------------------------
// Whole warp; the allocated column base is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- MMA ---------------------------------------------------------------------------
// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrives on the mbarrier once all previously issued MMAs of this thread completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// ---- fences --------------------------------------------------------------------------
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Ordinary shared-memory stores made visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- TMEM -> registers -------------------------------------------------------------------
// 16 consecutive FP32 columns of one lane per thread: warp w reads lanes 32 (w % 4) + lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// Hardware tanh approximation (one MUFU op).
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

}  // namespace tc
}  // namespace rw
