// PTX wrappers for the tensor-core (tcgen05 / TMEM) kernels: mbarriers with
// bounded waits, bulk async copies, UMMA descriptors and issue, TMEM loads.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace apsm {

enum GramMode : int { kBF16 = 0, kBF16x3 = 1, kTF32 = 2, kTF32x3 = 3 };

namespace tc {

// Operand format of a Gram mode: element type and the K extent of one UMMA
// (32 bytes); split modes carry a lo half after the hi half along K.
template <int MODE> struct OpTraits {
    static constexpr bool kTF = (MODE == kTF32 || MODE == kTF32x3);
    static constexpr bool kSplit = (MODE == kBF16x3 || MODE == kTF32x3);
    static constexpr int kElem = kTF ? 4 : 2;     // bytes per operand element
    static constexpr int kChunk = 16 / kElem;     // elements per 16-byte K chunk
    static constexpr int kStepK = 2 * kChunk;     // K per UMMA instruction (32 bytes)
};

// x = hi + lo with hi in the operand format (round to nearest) and lo the FP32 rest
template <int MODE> __device__ __forceinline__ void split_operand(float x, float* hi, float* lo)
{
    if constexpr (OpTraits<MODE>::kTF) {
        uint32_t h;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
        *hi = __uint_as_float(h);
    } else {
        *hi = __bfloat162float(__float2bfloat16_rn(x));
    }
    *lo = x - *hi;
}

// element (r, k) of a tile of R rows in the canonical K-major no-swizzle layout:
// byte (k / kc) * R * 16 + (r / 8) * 128 + (r % 8) * 16 + (k % kc) * elem
template <int MODE> __device__ __forceinline__ void put_operand(uint8_t* tile, int R, int r, int k, float v)
{
    using T = OpTraits<MODE>;
    uint8_t* p = tile + size_t(k / T::kChunk) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k % T::kChunk) * T::kElem;
    if constexpr (T::kTF) *reinterpret_cast<float*>(p) = v;
    else *reinterpret_cast<__nv_bfloat16*>(p) = __float2bfloat16_rn(v);
}

constexpr unsigned long long kWaitLimitNs = 2000000000ull; // bounded mbarrier waits (error instead of a hang)

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Non-blocking test of a barrier phase.
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Bounded wait (limit_ns, 2 s by default): false (and *abort set) when the
// barrier did not complete in time.  limit_ns == 0 gives up at once unless the
// phase is already complete (a test of the expiry path).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort,
                                          unsigned long long limit_ns = kWaitLimitNs)
{
    if (limit_ns == 0) {
        if (mbar_test_wait(bar, parity)) return true;
        *abort = 1;
        return false;
    }
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 64; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (*abort) return false;
        if (global_ns() - t0 > limit_ns) break;
    }
    *abort = 1;
    return false;
}

// Bounded wait used on the way out (also after an abort): in-flight async work
// must land before the CTA exits or releases tensor memory.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity)
{
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > kWaitLimitNs) return;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// UMMA shared-memory matrix descriptor, K-major, no swizzle ("interleaved"
// canonical layout): 8-row x 16-byte core matrices; lbo = byte distance of the
// two 16-byte K halves of one MMA K step, sbo = byte distance of 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(const void* base, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= uint64_t((smem_u32(base) >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46; // descriptor version for tcgen05
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor: FP32 accumulate, A/B K-major, M x N.
template <int MODE> __host__ __device__ constexpr uint32_t instr_desc(int M, int N)
{
    const uint32_t fmt = (MODE == kTF32 || MODE == kTF32x3) ? 2u : 1u; // TF32 : BF16
    return (1u << 4) | (fmt << 7) | (fmt << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

template <int MODE>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    if constexpr (MODE == kTF32 || MODE == kTF32x3) {
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
                     "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
    } else {
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
                     "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
    }
}

// The same with A in tensor memory (lane = row of A, one 32-bit column per K element for TF32):
// tmem_a is the column of A's first K element of this step.
template <int MODE>
__device__ __forceinline__ void umma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate)
{
    static_assert(MODE == kTF32 || MODE == kTF32x3, "A from tensor memory: TF32 operands only");
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
                 "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive 32-bit columns of this thread's TMEM lane (complete after tmem_st_wait).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]),
                 "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}

__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float ex2(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

} // namespace tc
} // namespace apsm
