// tcgen05.cuh — the fifth-generation tensor-core primitives used by the
// learned kernels, as inline PTX for sm_100a: tensor-memory allocation,
// shared-memory matrix descriptors (no-swizzle canonical layouts; callers OR
// a swizzle mode into bits 61-63 for the 32/64/128-byte swizzled layouts that
// TMA writes), BF16 x BF16 -> FP32 MMA issue, commit to an mbarrier,
// mbarrier waits and arrivals, TMA tiled loads and accumulator loads.
//
// Canonical no-swizzle layouts (one "core matrix" = 8 rows of 16 bytes):
//  * K-major operand (rows along M or N, K contiguous): element (r, k) of a
//    tile lives at  (r / 8) * SBO + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2
//    bytes from the tile base;
//  * MN-major operand (M or N contiguous): element (mn, k) lives at
//    (mn / 8) * SBO + (k / 8) * LBO + (k % 8) * 16 + (mn % 8) * 2.
// One MMA consumes K = 16 (two 8-wide K groups). Accumulator row i of an
// M = 128 tile is tensor-memory lane i; column j is column j.
#pragma once
#include <cstdint>

namespace nr {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor (SWIZZLE_NONE, version 1, base offset 0:
// the tensor cores apply a swizzle to the absolute address, as TMA does, so
// no base offset is needed for views that start inside a swizzle atom).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // descriptor version for sm_100
  return d;                 // layout type bits [61,64) = 0: no swizzle
}

// Instruction descriptor of tcgen05.mma kind::f16: BF16 A and B, FP32 D.
// a_mn / b_mn select MN-major operands.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N, bool a_mn, bool b_mn) {
  return (1u << 4)                       // D format: F32
         | (1u << 7)                     // A format: BF16
         | (1u << 10)                    // B format: BF16
         | ((a_mn ? 1u : 0u) << 15)      // A major
         | ((b_mn ? 1u : 0u) << 16)      // B major
         | ((N >> 3) << 17)              // N / 8
         | ((M >> 4) << 24);             // M / 16
}

// Allocates `ncols` (power of two >= 32) tensor-memory columns; the whole
// warp must call it. The base address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(smem_u32(dst)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols)
               : "memory");
}

// True in one lane of a converged warp (the lowest active one). MMA issue
// loops run on the whole warp, with descriptors that are the same in every
// lane, and only the elected lane issues: a loop run by one lane alone keeps
// its descriptors in per-thread registers and issued at less than half the
// rate in measurements on B200.
__device__ __forceinline__ bool elect_one() {
  uint32_t pred = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "elect.sync _|p, 0xffffffff;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(pred));
  return pred != 0;
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :: "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate) : "memory");
}

// Arrives once on the mbarrier when all MMAs issued so far by this thread
// have completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Makes this thread's generic-proxy shared-memory writes visible to the
// tensor cores (async proxy).
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Non-blocking test of a phase (mbarrier.test_wait): the cheap first probe
// when the phase has usually completed already (the blocking try_wait took
// some hundred cycles to report a completed phase in measurements on B200).
__device__ __forceinline__ bool mbar_test_now(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return done != 0;
}

// Waits for the phase with the given parity to complete; gives up after
// `limit` polls and returns false (the caller reports an error instead of
// hanging).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  if (mbar_test_now(bar, parity)) return true;
  const uint32_t a = smem_u32(bar);
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done) : "r"(a), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// Plain arrival (count 1) on an mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}
// Arrival that also announces `bytes` of bulk-copy transactions which must
// complete before the phase does.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Single poll of a phase; for waits that also watch an abort flag.
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return done != 0;
}

// Waits for `parity` on `bar`; gives up when `abort` is raised elsewhere, or
// after `limit` polls, when it raises `abort` itself. For kernels whose warps
// wait on one another's hand-overs: one failed wait releases them all. The
// first probe does not block; the later ones use the blocking try_wait
// (spinning on the non-blocking test was slower in measurements on B200).
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort,
                                                   uint32_t limit) {
  if (mbar_test_now(bar, parity)) return true;
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_test(bar, parity)) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}

// Tensor-memory-access (TMA) tiled loads from a tensor map in this GPU's
// global memory into this CTA's shared memory, completing on `bar` with the
// box's byte count. The destination is 128-byte aligned; the innermost
// coordinate c0 is always 0 here (16-byte aligned by construction).
__device__ __forceinline__ void tma_prefetch_map(const void* map) {
  asm volatile("prefetch.tensormap [%0];" :: "l"(reinterpret_cast<uint64_t>(map)) : "memory");
}
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];"
      :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
         "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const void* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
      :: "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
         "r"(smem_u32(bar))
      : "memory");
}

// Loads 8 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr) : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// The same load without the wait: the registers are valid only after
// tmem_wait_ld(), so several loads can be in flight at once.
__device__ __forceinline__ void tmem_ld8_nowait(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr) : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Byte offsets of the canonical layouts (see the file comment).
__host__ __device__ constexpr uint32_t kmajor_off(uint32_t r, uint32_t k, uint32_t lbo, uint32_t sbo) {
  return (r >> 3) * sbo + (k >> 3) * lbo + (r & 7u) * 16u + (k & 7u) * 2u;
}
__host__ __device__ constexpr uint32_t mnmajor_off(uint32_t mn, uint32_t k, uint32_t lbo, uint32_t sbo) {
  return (mn >> 3) * sbo + (k >> 3) * lbo + (k & 7u) * 16u + (mn & 7u) * 2u;
}

}  // namespace tc
}  // namespace nr
