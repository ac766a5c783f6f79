// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a, as inline PTX.
//
// Operands live in shared memory in the K-major, no-swizzle canonical layout: 8 x 8 blocks of
// 16-bit elements ("core matrices", 8 rows of 16 bytes, 128 contiguous bytes). A tile of R rows and
// K columns is stored row-group major, [R/8][K/8][8 rows][8 elements], so element (r, k) sits at byte
//     (r / 8) * (K / 8) * 128 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// In the shared-memory matrix descriptor the K-adjacent core matrices are 128 bytes apart (leading
// byte offset) and the row-group-adjacent ones K / 8 * 128 bytes apart (stride byte offset); one MMA
// consumes K = 16 (two core matrices) starting at the descriptor's address.
// Accumulators are FP32 in tensor memory: row i of an M = 128 tile is TMEM lane i, column j is TMEM
// column j. Every wait on an mbarrier is bounded by an iteration limit.
#pragma once

#include <cstdint>

namespace nwg {
namespace umma {

__device__ __forceinline__ std::uint32_t SmemAddress(const void *p) {
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) in a [R/8][K/8][8][8] 16-bit operand tile with K columns.
__host__ __device__ __forceinline__ std::uint32_t TileOffset(std::uint32_t r, std::uint32_t k, std::uint32_t K) {
    return (r >> 3) * (K >> 3) * 128u + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: K-major, no swizzle, version 1 (sm_100).
__device__ __forceinline__ std::uint64_t SmemDescriptor(std::uint32_t smem_address, std::uint32_t leading_bytes,
                                                        std::uint32_t stride_bytes) {
    std::uint64_t d = 0;
    d |= static_cast<std::uint64_t>((smem_address >> 4) & 0x3FFFu);
    d |= static_cast<std::uint64_t>((leading_bytes >> 4) & 0x3FFFu) << 16;
    d |= static_cast<std::uint64_t>((stride_bytes >> 4) & 0x3FFFu) << 32;
    d |= static_cast<std::uint64_t>(1u) << 46;  // descriptor version
    // base offset 0, leading-byte-offset mode 0, layout type 0 (no swizzle)
    return d;
}

// Instruction descriptor of kind::f16 with BF16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr std::uint32_t InstrDescBf16(int m, int n) {
    return (1u << 4)                                   // accumulator format: F32
           | (1u << 7)                                 // A format: BF16
           | (1u << 10)                                // B format: BF16
           | (static_cast<std::uint32_t>(n >> 3) << 17)
           | (static_cast<std::uint32_t>(m >> 4) << 24);
}

// Warp-collective: allocate `columns` (power of two >= 32) TMEM columns; the base address is written
// to *holder (shared memory).
__device__ __forceinline__ void Alloc(std::uint32_t *holder, std::uint32_t columns) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddress(holder)),
                 "r"(columns));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void Dealloc(std::uint32_t base, std::uint32_t columns) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(columns));
}

__device__ __forceinline__ void FenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void FenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Makes generic-proxy shared-memory writes visible to the tensor core (async proxy).
__device__ __forceinline__ void FenceProxyAsyncShared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] x B[smem]^T, issued by one thread.
__device__ __forceinline__ void Mma(std::uint32_t tmem_d, std::uint64_t a_desc, std::uint64_t b_desc,
                                    std::uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u));
}

// D[tmem] (+)= A[tmem] x B[smem]^T with the A operand in tensor memory: row i of A in lane i, two 16-bit
// elements per 32-bit column in ascending K order (the lower element in the low half), issued by one thread.
__device__ __forceinline__ void MmaTs(std::uint32_t tmem_d, std::uint32_t tmem_a, std::uint64_t b_desc,
                                      std::uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u));
}

// Arrive on the mbarrier once every previously issued MMA of this thread has completed.
__device__ __forceinline__ void Commit(std::uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     SmemAddress(mbar))
                 : "memory");
}

__device__ __forceinline__ void MbarInit(std::uint64_t *mbar, std::uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddress(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Whether the mbarrier phase with the given parity has completed (non-blocking).
__device__ __forceinline__ bool MbarTest(std::uint64_t *mbar, std::uint32_t parity) {
    std::uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(SmemAddress(mbar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits for the mbarrier phase with the given parity; gives up after `limit` polls, or as soon as another thread
// of the CTA has recorded a failure in *failed (checked every 16 polls), and returns false.
__device__ __forceinline__ bool MbarWaitOrStop(std::uint64_t *mbar, std::uint32_t parity, std::uint32_t limit,
                                               const int *failed) {
    if (MbarTest(mbar, parity)) {
        return true;
    }
    const std::uint32_t addr = SmemAddress(mbar);
    for (std::uint32_t i = 0; i < limit; ++i) {
        if ((i & 15u) == 0u && *reinterpret_cast<const volatile int *>(failed) != 0) {
            return false;
        }
        std::uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) {
            return true;
        }
    }
    return false;
}

// Waits for the mbarrier phase with the given parity; gives up after `limit` polls and returns false.
// A phase that has completed already is seen by the non-blocking test_wait; the potentially blocking try_wait
// took hundreds of cycles to report such a phase on B200, so it is used only while the phase is still open.
__device__ __forceinline__ bool MbarWait(std::uint64_t *mbar, std::uint32_t parity, std::uint32_t limit) {
    if (MbarTest(mbar, parity)) {
        return true;
    }
    const std::uint32_t addr = SmemAddress(mbar);
    for (std::uint32_t i = 0; i < limit; ++i) {
        std::uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) {
            return true;
        }
    }
    return false;
}

// Writes 16 consecutive 32-bit columns of this thread's TMEM lane (warp w writes lanes 32w..32w+31); WaitStore
// makes them visible before a later tensor-core read.
__device__ __forceinline__ void Store16(std::uint32_t taddr, const std::uint32_t (&r)[16]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
                 : "memory");
}

__device__ __forceinline__ void WaitStore() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31).
__device__ __forceinline__ void Load32(std::uint32_t taddr, float (&v)[32]) {
    std::uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

// 64 consecutive FP32 accumulator columns of this thread's TMEM lane in one load and one wait.
__device__ __forceinline__ void Load64(std::uint32_t taddr, float (&v)[64]) {
    std::uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) {
        v[i] = __uint_as_float(r[i]);
    }
}

}  // namespace umma
}  // namespace nwg
