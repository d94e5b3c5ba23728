// umma.cuh — thin device wrappers for the sm_100a tensor-core path: TMA tile
// loads, mbarriers with bounded waits, TMEM allocation, tcgen05.mma issue and
// commit, and TMEM -> register loads.
//
// Operand convention used throughout: both GEMM operands are K-major bf16
// tiles of 128 rows x 64 elements (128 bytes per row), written by TMA with the
// 128-byte swizzle.  In that canonical layout eight rows form one 1024-byte
// swizzle atom, so the shared-memory matrix descriptor has
//   stride byte offset (between 8-row groups) = 1024 B,
//   leading byte offset = 16 B (unused for swizzled K-major),
//   layout = SWIZZLE_128B, version = 1 (sm_100),
// and the k-th 16-element slice of the 64-element row starts 32 * k bytes
// further (the hardware applies the swizzle to the final address, so the
// tile base must be 1024-byte aligned).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pfb {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// ------------------------------------------------------------------ mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
            smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

// Wait for the phase with the given parity to complete.  Gives up after
// `limit` polls (each poll may block for a short hardware-defined time) and
// returns false, so a broken pipeline ends the kernel instead of hanging it.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          uint32_t limit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// As mbar_wait, but also gives up as soon as *abort is nonzero (another role
// of the CTA has failed), so one failed wait does not leave the others
// polling until their own limits run out.
__device__ __forceinline__ bool mbar_wait_abort(uint64_t* bar, uint32_t parity,
                                                uint32_t limit,
                                                const volatile int* abort) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (*abort) return false;
    }
    return false;
}

// One plain arrival on the mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ------------------------------------------------------------------ TMA
// 2-D tiled load of the box at element coordinates (x = inner, y = row) into
// shared memory, completing `bytes` on the mbarrier.  x * 2 bytes must be a
// multiple of 16 (callers use multiples of 64 elements).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map,
                                            uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::"
        "complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y),
        "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
}

// ------------------------------------------------------------------ TMEM
// Warp-wide: allocate `ncols` (power of two >= 32) TMEM columns; the base
// address is written to shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
            smem_u32(slot)),
        "r"(ncols)
        : "memory");
}

__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::
                     : "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(
                     taddr),
                 "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// ------------------------------------------------------------------ MMA
// Instruction descriptor of kind::f16 with bf16 A and B (the same type for
// both operands), f32 accumulation, both operands K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4)                      // D format: f32
           | (1u << 7)                    // A format: bf16
           | (1u << 10)                   // B format: bf16
           | ((uint32_t)(N >> 3) << 17)   // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled tile whose
// rows are 128 bytes apart (see the header comment).
__device__ __forceinline__ uint64_t desc_kmajor_sw128(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu)   // start address / 16
           | ((uint64_t)1u << 16)               // leading byte offset 16 B
           | ((uint64_t)(1024u >> 4) << 32)     // stride byte offset 1024 B
           | ((uint64_t)1u << 46)               // descriptor version (sm_100)
           | ((uint64_t)2u << 61);              // SWIZZLE_128B
}

// D[tmem] (+)= A[smem] * B[smem]^T for one 128 x N x 16 step.  Issued by one
// thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc,
                                         uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive once on the mbarrier when all previously issued tcgen05 operations
// of this thread have completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
        "[%0];" ::"r"(smem_u32(bar))
        : "memory");
}

// Warp-wide: 32 consecutive f32 columns of the warp's 32 TMEM lanes (lane i
// of the warp receives row i of its lane quarter).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
          "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace umma
}  // namespace pfb
