// Thin wrappers over the sm_100a PTX used by the tensor-core kernels:
// mbarriers, 1-D bulk copies (global -> shared), tcgen05 MMA / TMEM.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mshqc_cd {
namespace sm100 {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarrier ------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
    return t;
}
// Bounded wait: gives up after `limit_ns` of wall time and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (true) {
#pragma unroll 1
        for (int k = 0; k < 256; ++k)
            if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// Relaxed GPU-scope loads and stores of an int shared between CTAs (progress
// counters that order nothing the results depend on).
__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(int* p, int v) {
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// dst[0..7] (+)= (double)src[0..7] as one ordered block of 16-byte accesses
// (dst 16-byte aligned).  As inline PTX the compiler keeps the block in
// place, so the 8 conversions of one block are live at a time instead of
// being hoisted over a whole tile row.
__device__ __forceinline__ void f32x8_to_f64(double* dst, const float* src, bool accumulate) {
    if (accumulate)
        asm volatile(
            "{\n\t.reg .f64 x<8>, y<8>;\n\t"
            "ld.global.v2.f64 {x0, x1}, [%0];\n\t"
            "ld.global.v2.f64 {x2, x3}, [%0+16];\n\t"
            "ld.global.v2.f64 {x4, x5}, [%0+32];\n\t"
            "ld.global.v2.f64 {x6, x7}, [%0+48];\n\t"
            "cvt.f64.f32 y0, %1;\n\tcvt.f64.f32 y1, %2;\n\tcvt.f64.f32 y2, %3;\n\tcvt.f64.f32 y3, %4;\n\t"
            "cvt.f64.f32 y4, %5;\n\tcvt.f64.f32 y5, %6;\n\tcvt.f64.f32 y6, %7;\n\tcvt.f64.f32 y7, %8;\n\t"
            "add.rn.f64 x0, x0, y0;\n\tadd.rn.f64 x1, x1, y1;\n\tadd.rn.f64 x2, x2, y2;\n\tadd.rn.f64 x3, x3, y3;\n\t"
            "add.rn.f64 x4, x4, y4;\n\tadd.rn.f64 x5, x5, y5;\n\tadd.rn.f64 x6, x6, y6;\n\tadd.rn.f64 x7, x7, y7;\n\t"
            "st.global.v2.f64 [%0], {x0, x1};\n\t"
            "st.global.v2.f64 [%0+16], {x2, x3};\n\t"
            "st.global.v2.f64 [%0+32], {x4, x5};\n\t"
            "st.global.v2.f64 [%0+48], {x6, x7};\n\t"
            "}\n" ::"l"(dst),
            "f"(src[0]), "f"(src[1]), "f"(src[2]), "f"(src[3]), "f"(src[4]), "f"(src[5]), "f"(src[6]), "f"(src[7])
            : "memory");
    else
        asm volatile(
            "{\n\t.reg .f64 y<8>;\n\t"
            "cvt.f64.f32 y0, %1;\n\tcvt.f64.f32 y1, %2;\n\tcvt.f64.f32 y2, %3;\n\tcvt.f64.f32 y3, %4;\n\t"
            "cvt.f64.f32 y4, %5;\n\tcvt.f64.f32 y5, %6;\n\tcvt.f64.f32 y6, %7;\n\tcvt.f64.f32 y7, %8;\n\t"
            "st.global.v2.f64 [%0], {y0, y1};\n\t"
            "st.global.v2.f64 [%0+16], {y2, y3};\n\t"
            "st.global.v2.f64 [%0+32], {y4, y5};\n\t"
            "st.global.v2.f64 [%0+48], {y6, y7};\n\t"
            "}\n" ::"l"(dst),
            "f"(src[0]), "f"(src[1]), "f"(src[2]), "f"(src[3]), "f"(src[4]), "f"(src[5]), "f"(src[6]), "f"(src[7])
            : "memory");
}

// Wave pacing of a persistent kernel whose CTAs share operands through L2.
// The CTAs of one wave of tiles read the same operand slabs; if they stay
// within a few microseconds of each other, every slab comes from DRAM once
// and serves all of them from L2.  Left alone they drift apart, L2 evicts a
// slab before its last reader arrives, the misses raise the DRAM fill rate
// and shorten what L2 keeps, and the drift feeds itself.  The producer warp of
// each CTA counts the copies it issues; every `every` copies it publishes
// its epoch in prog[cta] and waits until every CTA has published at least
// epoch - slack.  The slowest CTA's own condition always holds, so every wait
// ends while all CTAs are resident; a wait that runs past limit_ns (a CTA not
// resident because another kernel holds its SM) turns pacing off for the rest
// of the launch.  Pacing orders no data the results depend on.  All 32 lanes
// of the producer warp call step() together.
struct WavePacer {
    int* prog;
    int ncta, every, slack, cnt;
    bool on;
    __device__ void init(int* p, int n, int ev, int sl) {
        prog = p;
        ncta = n;
        every = ev > 0 ? ev : 1;
        slack = sl;
        cnt = 0;
        on = p != nullptr;
    }
    __device__ void step(int lane, uint64_t limit_ns) {
        if (!on) return;
        if (cnt % every == 0) {
            const int e = cnt / every;
            if (lane == 0) st_relaxed_gpu(prog + blockIdx.x, e);
            if (e > slack) {
                const int target = e - slack;
                uint64_t t0 = globaltimer_ns();
                t0 = __shfl_sync(0xffffffffu, t0, 0);
                while (true) {
                    bool ok = true;
                    for (int c = lane; c < ncta; c += 32) ok &= ld_relaxed_gpu(prog + c) >= target;
                    if (__all_sync(0xffffffffu, ok)) break;
                    uint64_t dt = globaltimer_ns() - t0;
                    dt = __shfl_sync(0xffffffffu, dt, 0);
                    if (dt > limit_ns) {
                        on = false;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        ++cnt;
    }
    // this CTA issues no more copies: nobody waits for it
    __device__ void finish(int lane) {
        if (prog && lane == 0) st_relaxed_gpu(prog + blockIdx.x, 0x7fffffff);
    }
};

// Named barrier `id` over `nthreads` threads that also returns whether ANY of
// them passed pred = true, so a group of warps leaves a loop together.
__device__ __forceinline__ bool bar_any(int id, int nthreads, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, %2, %3, q;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// ---- 1-D bulk copy (no multicast) -----------------------------------------
// dst / src 16-byte aligned, bytes a multiple of 16; completion counted on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// ---- tcgen05 ----------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_addr(slot_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (16-bit inputs, type in idesc), one thread.
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// D[tmem] (+)= A * B^T, signed 8-bit integers, exact 32-bit integer accumulation
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive on bar once all previously issued tcgen05 ops of this thread completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
            smem_addr(bar))
        : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns per warp.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
// 32 lanes x 16 consecutive 32-bit columns per warp.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
template <int W>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[W]) {
    if constexpr (W == 32)
        tmem_ld32(taddr, r);
    else
        tmem_ld16(taddr, r);
}
__device__ __forceinline__ void tmem_ld_wait() {
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Instruction descriptor, kind::f16: FP16 x FP16 -> FP32, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_f16_f32(int M, int N) {
    return (1u << 4)                        // D format: F32; A, B format 0: F16
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(M >> 4) << 24);    // M / 16
}

// Instruction descriptor, kind::i8: S8 x S8 -> S32, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_s8_s32(int M, int N) {
    return (2u << 4)                        // D format: S32
           | (1u << 7)                      // A format: signed 8-bit
           | (1u << 10)                     // B format: signed 8-bit
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(M >> 4) << 24);    // M / 16
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4)                        // D format: F32
           | (1u << 7)                      // A format: BF16
           | (1u << 10)                     // B format: BF16
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(M >> 4) << 24);    // M / 16
}

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of
// 8 rows x 16 bytes; lbo = byte distance between the two core matrices of one
// K=16 slice, sbo = byte distance between consecutive 8-row groups.
__device__ __forceinline__ uint64_t smem_desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version (sm_100)
    // base offset 0, lbo mode 0, layout type 0 (no swizzle)
    return d;
}

// 1/D in FP64 from the FP32 hardware reciprocal seed and one Newton-Raphson
// step r <- r + r (1 - D r) (relative error ~ (2^-22)^2).
__device__ __forceinline__ double recip_nr(double D) {
    float df = (float)D;
    float r0;
    asm("rcp.approx.ftz.f32 %0, %1;\n" : "=f"(r0) : "f"(df));
    double r = (double)r0;
    double e = fma(-D, r, 1.0);
    r = fma(r, e, r);
    e = fma(-D, r, 1.0);
    return fma(r, e, r);
}

}  // namespace sm100
}  // namespace mshqc_cd
