// Blackwell (sm_100a) tensor-core building blocks in inline PTX: shared
// memory matrix descriptors, the tcgen05 instruction descriptor for
// BF16 x BF16 -> FP32, tcgen05.mma / commit / ld, TMEM allocation, mbarriers
// with bounded waits and cp.async staging.
//
// Shared-memory operand layout (no swizzle). A 16 B row of 8 BF16 values is
// the unit; 8 such rows (128 B, contiguous) form a core matrix. For a
// K-major operand (rows = M or N, K contiguous in 16 B rows) element (r, k)
// lives at
//     (r % 8) * 16 + (r / 8) * SBO + (k % 8) * 2 + (k / 8) * LBO
// and for an MN-major operand (8 consecutive rows contiguous in 16 B) at
//     (r % 8) * 2 + (r / 8) * SBO + (k % 8) * 16 + (k / 8) * LBO.
// In both cases SBO is the byte stride between groups of 8 rows and LBO the
// byte stride between groups of 8 K values; one K=16 MMA reads two K groups.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_bf16.h>

namespace crt {
namespace tc {

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared memory descriptor: start address, LBO and SBO in 16 B units,
// version 1 (sm_100), base offset 0, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;  // descriptor version
    return d;
}

// Descriptor of a K-major operand in one of the swizzled layouts that TMA
// writes (rows of `row_bytes` = 32, 64 or 128 B, 16 B chunks XOR-permuted
// by address bits 7.. of the row): SBO = 8 rows, LBO unused, base offset 0.
// The hardware swizzles on absolute shared-memory addresses, so the start
// may sit any whole number of rows (and 32 B K-steps) into a swizzle atom.
// For an MN-major operand in the same layouts (rows of the K dimension, each
// holding row_bytes of consecutive M or N elements), lbo_bytes is the stride
// between such groups of M / N elements.
__device__ __forceinline__ uint64_t smem_desc_sw(uint32_t addr, uint32_t row_bytes, uint32_t lbo_bytes = 16) {
    const uint64_t layout = row_bytes == 128 ? 2 : row_bytes == 64 ? 4 : 6;
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)(((8 * row_bytes) >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    d |= layout << 61;
    return d;
}

// Instruction descriptor of kind::f16 with BF16 A/B and FP32 D, M x N tile;
// a_mn / b_mn select MN-major operands.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4)                        // D format F32
           | (1u << 7)                      // A format BF16
           | (1u << 10)                     // B format BF16
           | ((a_mn ? 1u : 0u) << 15)       // A major
           | ((b_mn ? 1u : 0u) << 16)       // B major
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(M >> 4) << 24);    // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// The same, executed by a whole converged warp: one lane (elect.sync)
// issues. Running the issue loop warp-uniformly lets the compiler keep the
// descriptors in uniform registers; a loop under `if (lane == 0)` pays
// register moves per MMA and issues far slower.
__device__ __forceinline__ void mma_bf16_warp(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
    asm volatile(
        "{\n\t"
        ".reg .pred p, e;\n\t"
        "elect.sync _|e, 0xffffffff;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}
__device__ __forceinline__ void mma_commit_warp(uint32_t mbar) {
    asm volatile(
        "{\n\t"
        ".reg .pred e;\n\t"
        "elect.sync _|e, 0xffffffff;\n\t"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n\t"
        "}\n" ::"r"(mbar)
        : "memory");
}

// Arrives on the mbarrier once every tcgen05.mma issued so far by this
// thread has completed.
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes visible to the async proxy (MMA reads).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation by one full warp; the base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32w..32w+31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Waits for the completion of phase `parity` of the mbarrier; gives up
// after `limit` polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = 1u << 24) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Same, but also gives up as soon as *abort is set by another thread of the
// block (which then stops waiting on this block's other barriers too); on a
// timeout it sets *abort itself.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, uint32_t parity, volatile int *abort) {
    for (int round = 0; round < 256; ++round) {
        if (*abort) return false;
        if (mbar_wait(bar, parity, 1u << 16)) return true;
    }
    *abort = 1;
    return false;
}

// Warp-uniform form of mbar_wait_or_abort for a converged warp: lane 0's
// outcome is everyone's.
__device__ __forceinline__ bool mbar_wait_or_abort_warp(uint64_t *bar, uint32_t parity, volatile int *abort) {
    bool ok = false;
    if ((threadIdx.x & 31) == 0) ok = mbar_wait_or_abort(bar, parity, abort);
    return __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
}

// Plain arrive (release at CTA scope) by this thread.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile(
        "{\n\t"
        ".reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t"
        "}\n" ::"r"(smem_addr(bar))
        : "memory");
}

// Arrive and add `bytes` to the transaction count the phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile(
        "{\n\t"
        ".reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t"
        "}\n" ::"r"(smem_addr(bar)),
        "r"(bytes)
        : "memory");
}

// TMA tiled loads (no multicast) into this CTA's shared memory; completion
// is signalled as transaction bytes on the mbarrier. Coordinates are
// elements, innermost first; out-of-bounds elements are filled with zeros.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// Named barrier `id` (1..15) over `nthreads` threads (a multiple of 32).
__device__ __forceinline__ void named_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// 16 B global -> shared copy; src_bytes = 0 fills zeros (src must still be
// a valid address).
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

#endif  // __CUDACC__

}  // namespace tc
}  // namespace crt
