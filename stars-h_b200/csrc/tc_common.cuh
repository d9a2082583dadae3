// tcgen05 / mbarrier / TMA helpers shared by the tensor-core kernels
// (sketch_i8.cu, gen_sketch_i8.cu).  Inline PTX for sm_100a.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cudaTypedefs.h>

namespace b200 {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory descriptor of a K-major operand without swizzle:
// core matrices of 8 rows x 16 bytes (128 contiguous bytes), lbo = byte
// distance between the two 16-byte K halves of one MMA, sbo = byte
// distance between consecutive 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo,
                                              uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;            // descriptor version (sm_100)
    return d;                          // base offset 0, no swizzle
}

// Instruction descriptor of kind::i8: int32 accumulator, int8 A (unsigned
// digits, or a signed top digit), signed int8 B, both K-major, M = m
// (64 or 128), N = n (multiple of 16 up to 256).
__host__ __device__ constexpr uint32_t idesc_i8_mn(int m, int n, bool a_signed)
{
    return (2u << 4) | ((a_signed ? 1u : 0u) << 7) | (1u << 10) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da,
                                       uint64_t db, uint32_t idesc,
                                       int accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

// Arrives (once) on mbar when every MMA this thread issued so far is done.
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)));
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                 :: "r"(smem_u32(mbar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint64_t *mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred P1;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(mbar)), "r"(parity) : "memory");
    return ok != 0;
}

// Waits for the completion of the phase of the given parity; gives up
// after about two seconds, or as soon as *abort is set by another thread,
// and returns false.
__device__ __forceinline__ bool mbar_wait_or(uint64_t *mbar, uint32_t parity,
                                             volatile int *abort)
{
    const long long t0 = clock64();
    while (!mbar_try(mbar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > (1ll << 32)) return false;
    }
    return true;
}

// As mbar_wait_or, for roles that wait long stretches (epilogues, the MMA
// and staging warps of the compute-bound kernels): between polls the warp
// sleeps about `ns` nanoseconds, leaving the issue slots to the warps that
// compute.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t *mbar, uint32_t parity,
                                                volatile int *abort,
                                                unsigned ns)
{
    const long long t0 = clock64();
    while (!mbar_try(mbar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > (1ll << 32)) return false;
        __nanosleep(ns);
    }
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(mbar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]),
                   "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

// TMA tile copy (this CTA only) of a 3-D box at (c0, c1, c2); completes on
// mbar.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map,
                                            int c0, int c1, int c2,
                                            uint64_t *mbar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1, {%2, %3, %4}], [%5];"
                 :: "r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2),
                    "r"(smem_u32(mbar))
                 : "memory");
}

// TMA tile copy (this CTA only) of a 2-D box at (c0, c1); completes on mbar.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map,
                                            int c0, int c1, uint64_t *mbar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1, {%2, %3}], [%4];"
                 :: "r"(smem_u32(dst)), "l"(map), "r"(c0), "r"(c1),
                    "r"(smem_u32(mbar))
                 : "memory");
}

// Bulk copy (no tensor map) of `bytes` bytes from global to this CTA's
// shared memory; both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src,
                                          uint32_t bytes, uint64_t *mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;"); }

// Named barrier over `count` threads (a multiple of 32), id 1..15.
__device__ __forceinline__ void named_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(count) : "memory");
}

// Tensor-map encoder from the driver (cuTensorMapEncodeTiled), or null.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// Tensor map of an int8 matrix stored column-major (ld rows per column,
// `cols` columns) with a 16 x nc box; columns past `cols` read as zero.
bool i8_colmajor_map(CUtensorMap *map, const int8_t *base, int ld, int cols,
                     int nc);

}  // namespace b200
