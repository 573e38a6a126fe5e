// soapb_tc.cuh -- fifth-generation tensor cores (tcgen05) for the site kernels.
//
// The contractions run as kind::tf32 MMAs with FP32 accumulators in tensor
// memory (TMEM).  Operands live in shared memory in the K-major layout without
// swizzling: a tile of R rows by KT 32-bit elements is cut into 8-row x 16-byte
// core matrices, the core matrices of one 8-row group consecutive along K
// (LBO = 128 bytes), the 8-row groups one after the other (SBO = KT/4 x 128
// bytes).  One MMA consumes K = 8 elements (two core matrices along K); the
// next K-step starts 256 bytes further on.
//
// Precision: 3xTF32.  Each FP32 operand is split into a TF32 head and the
// TF32 rounding of its remainder, a = a_hi + a_lo to ~22 bits, and a b is
// taken as a_lo b_hi + a_hi b_lo + a_hi b_hi (the small terms first) into the
// same FP32 accumulator -- the product's error is then ~2^-22 relative, close
// to an FP32 multiply.
//
// Synchronisation: threads write operands with ordinary stores, then
// fence.proxy.async makes them visible to the tensor core's (async) proxy; one
// elected thread issues the MMAs and a tcgen05.commit that arrives on an
// mbarrier when they complete; every thread waits on that mbarrier (a bounded
// wait: a wait that gives up reports an error) before reading TMEM.
#pragma once

#include <cstdint>

namespace soapb {
namespace tc {

constexpr int kLBO = 128;
// polls of an mbarrier before a wait gives up (each poll may itself block for
// a short, hardware-defined time)
constexpr int kMaxTries = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in a K-major, unswizzled tile of KT columns.
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int KT) {
  return (uint32_t)((r >> 3) * (KT >> 2) * 128 + (k >> 2) * kLBO + (r & 7) * 16 + (k & 3) * 4);
}

// Shared-memory matrix descriptor: start address, LBO, SBO (all >> 4), the
// sm_100 descriptor version (bit 46), no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, int KT) {
  const uint32_t sbo = (uint32_t)(KT >> 2) * 128;
  uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)(kLBO >> 4) << 16;
  d |= (uint64_t)(sbo >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::tf32, FP32 accumulator, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// x = hi + lo with both parts TF32-representable (as 32-bit patterns)
__device__ __forceinline__ void split(float x, uint32_t &hi, uint32_t &lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

// ---- TMEM allocation (one warp) -------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- fences ------------------------------------------------------------------
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- MMA and its completion --------------------------------------------------
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{.reg .pred p; setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(mbar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t *mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for the phase with parity `parity` to complete; gives up after
// max_tries polls (each poll may itself block for a short, hardware-defined
// time).  Returns 1 when the phase completed.
__device__ __forceinline__ int mbar_wait(uint64_t *mbar, uint32_t parity, int max_tries) {
  uint32_t done = 0;
  for (int it = 0; it < max_tries && !done; ++it)
    asm volatile(
        "{.reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p;}"
        : "=r"(done)
        : "r"(smem_addr(mbar)), "r"(parity)
        : "memory");
  return (int)done;
}

// 3xTF32 product of two split operands into one accumulator, K = 8 per step.
// a_hi/a_lo/b_hi/b_lo: tile bases in shared memory; KTa/KTb their K widths;
// k0: the first K column (multiple of 8).
__device__ __forceinline__ void mma3_step(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo, int KTa, uint32_t b_hi,
                                          uint32_t b_lo, int KTb, int k0, uint32_t idesc, uint32_t accumulate) {
  const uint32_t oa = (uint32_t)(k0 >> 2) * kLBO, ob = (uint32_t)(k0 >> 2) * kLBO;
  mma_tf32(d_tmem, smem_desc(a_lo + oa, KTa), smem_desc(b_hi + ob, KTb), idesc, accumulate);
  mma_tf32(d_tmem, smem_desc(a_hi + oa, KTa), smem_desc(b_lo + ob, KTb), idesc, 1u);
  mma_tf32(d_tmem, smem_desc(a_hi + oa, KTa), smem_desc(b_hi + ob, KTb), idesc, 1u);
}

// ---- TMEM -> registers: 32 lanes x 16 columns, one row per thread ------------
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// TMEM address of lane `lane`, column `col` relative to a base from tmem_alloc.
__device__ __forceinline__ uint32_t taddr(uint32_t base, int lane, int col) {
  return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

}  // namespace tc
}  // namespace soapb
