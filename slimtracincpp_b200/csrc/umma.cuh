// Blackwell (sm_100a) tensor-core primitives used by the radiance-cache MLP:
// tcgen05.mma kind::f16 (bf16 operands in shared memory, f32 accumulator in
// tensor memory), TMEM allocation and loads, and bounded mbarrier waits.
//
// Operand images.  Every bf16 matrix in shared memory is stored as a grid of
// "core matrices" of 8 rows x 16 bytes (8 bf16), 128 contiguous bytes each,
// with no swizzle.  For an R-row x C-column matrix the byte offset of element
// (r, c) is
//     (c / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (c % 8) * 2
// i.e. the 16-byte row pieces of one column group are contiguous, column
// groups follow each other.  One image serves two operand roles:
//   K-major   rows are M (or N), columns are K:  LBO = R*16 (next 8 K),
//             SBO = 128 (next 8 rows); a K=16 step advances 2*R*16 bytes.
//   MN-major  rows are K, columns are M (or N):  LBO = 128 (next 8 K rows),
//             SBO = R*16 (next 8 columns); a K=16 step advances 256 bytes.
// So the sample-major activation tiles written for the forward pass are read
// back unchanged, MN-major, as the operands of the weight-gradient GEMMs,
// and the weight images are read MN-major for the input-gradient GEMMs.
//
// TMEM accumulators: an M=128 MMA writes row m to lane m; an M=64 MMA writes
// row m to lane (m % 16) + 32 * (m / 16), so warp w (lanes 32w..32w+31) holds
// rows 16w..16w+15 in its first 16 lanes.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace slim {
namespace umma {

#define SLIM_U __device__ __forceinline__

SLIM_U uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (sm_100 version 1, no swizzle).
SLIM_U uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// Operand at K step `k` (K = 16 per MMA) of an image with `rows` rows.
SLIM_U uint64_t kmajor(uint32_t base, uint32_t rows, uint32_t k) {
    return desc(base + k * 2u * rows * 16u, rows * 16u, 128u);
}
SLIM_U uint64_t mnmajor(uint32_t base, uint32_t rows, uint32_t k) {
    return desc(base + k * 256u, 128u, rows * 16u);
}

// Instruction descriptor: bf16 x bf16 -> f32, dense.
constexpr uint32_t idesc_bf16(int M, int N, int a_mn_major, int b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn_major << 15) | ((uint32_t)b_mn_major << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

SLIM_U void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                 ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
// Arrive on `bar` once every MMA this thread issued so far has completed.
SLIM_U void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_addr(bar)) : "memory");
}

SLIM_U void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
SLIM_U bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Wait for phase `parity` of `bar` to complete, giving up after about a
// second (2^31 SM cycles); returns false on timeout.
SLIM_U bool mbar_wait(uint64_t *bar, uint32_t parity) {
    long long t0 = clock64();
    while (!mbar_try(bar, parity))
        if (clock64() - t0 > (1ll << 31)) return false;
    return true;
}

// TMEM allocation (one whole warp executes these).
SLIM_U void tmem_alloc(uint32_t *dst_smem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
                 "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
SLIM_U void tmem_free(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's lane (warp-wide).
SLIM_U void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
SLIM_U void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Ordering around thread barriers and between the generic and async proxies.
SLIM_U void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
SLIM_U void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
SLIM_U void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM address of lane `lane`, column `col`, relative to an allocation base.
SLIM_U uint32_t tmem_at(uint32_t base, uint32_t lane, uint32_t col) { return base + (lane << 16) + col; }

#undef SLIM_U

}  // namespace umma
}  // namespace slim
