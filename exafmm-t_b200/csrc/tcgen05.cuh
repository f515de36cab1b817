// sm_100a tensor-core primitives (PTX ISA 8.6+ tcgen05 family) used by the M2L Hadamard kernel:
// tensor-memory (TMEM) allocation, register <-> TMEM moves, the single-thread-issued MMA with its
// operand A in TMEM and B in shared memory, completion through an mbarrier, and the fences that
// order them against ordinary thread synchronisation.
#pragma once
#include <cstdint>

namespace xfmm {
namespace tc5 {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// One lane of the (converged) warp gets true.  The MMAs below are issued this way, by an elected lane of
// a converged warp with warp-uniform operands: issued from a single thread of a divergent branch they
// cost an order of magnitude more issue time each.
__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile("{\n\t.reg .pred px;\n\telect.sync _|px, 0xffffffff;\n\tselp.b32 %0, 1, 0, px;\n\t}" : "=r"(pred));
  return pred != 0;
}

// ---- TMEM allocation (one full warp executes each of these)
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- ordering of tcgen05 operations across thread synchronisation
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// generic-proxy shared-memory writes made visible to the tensor core's (async-proxy) reads
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- register <-> TMEM, shape 32x32b repeated 16 times: lane i of the warp moves 16 consecutive
// 32-bit columns of TMEM lane (lane field of taddr) + i.  A warp reaches only its own quarter of the
// 128 lanes (warp w % 4 -> lanes 32 (w % 4) .. +31).
__device__ __forceinline__ void st_32x32b_x16(uint32_t taddr, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}
// shape 16x256b repeated twice: a 16-lane x 16-column block; lane t of the warp (g = t / 4, q = t % 4)
// moves v[0..1] to (lane g, columns 2q, 2q + 1), v[2..3] to (lane g + 8, 2q, 2q + 1), v[4..5] to
// (lane g, 8 + 2q, 9 + 2q) and v[6..7] to (lane g + 8, 8 + 2q, 9 + 2q), lanes relative to taddr's lane
__device__ __forceinline__ void st_16x256b_x2(uint32_t taddr, const uint32_t (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.16x256b.x2.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
               "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}
__device__ __forceinline__ void ld_32x32b_x16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}

// ---- MMA, D (TMEM, FP32) (+)= A (TMEM, TF32, K-major) x B (shared memory, TF32), issued by one thread
__device__ __forceinline__ void mma_tf32_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// the mbarrier at mbar (shared address) receives one arrival when every MMA this thread issued so far
// has completed
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// Instruction descriptor of kind::tf32 with FP32 accumulation, A and B K-major, shape M x N
// (bits 4-5 D format, 7-9 A format, 10-12 B format, 15/16 A/B major, 17-22 N / 8, 24-28 M / 16).
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
// Shared-memory matrix descriptor, no swizzle: the operand is a grid of core matrices of 8 rows x 16 bytes
// (each 128 contiguous bytes, row r at 16 r); lbo = bytes between the core matrices adjacent along K,
// sbo = bytes between those adjacent along M / N.  Bits 46-47 hold the descriptor version (1 on sm_100).
__device__ __forceinline__ uint64_t sdesc_nosw(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}

// ---- per-thread asynchronous global -> shared copies of 16 bytes (src_bytes 0: the 16 bytes are zeroed)
__device__ __forceinline__ void cp_async16(uint32_t dst_smem, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst_smem), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {  // at most N of this thread's groups still in flight
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- mbarrier
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(mbar) : "memory");
}
// one arrival that also expects `bytes` of asynchronous copies to complete on this phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(mbar),
               "r"(bytes)
               : "memory");
}
// bulk copy global -> this CTA's shared memory (no multicast); both addresses 16-byte aligned, bytes a
// multiple of 16; completion is counted in bytes on the mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst_smem, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst_smem),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
// try_wait that lets the hardware suspend the thread until the phase completes or about `ns` pass
__device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t mbar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(mbar), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete, for at most `limit` SM clock cycles; false if it
// did not complete in time.  Each try suspends the thread (up to a millisecond) instead of spinning.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long long limit) {
  if (mbar_try_wait(mbar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait_sleep(mbar, parity, 1000000u))
    if (clock64() - t0 > limit) return false;
  return true;
}

}  // namespace tc5
}  // namespace xfmm
