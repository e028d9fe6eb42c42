// Common device helpers for the Cholesky-MP2 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mshqc_cd {

constexpr double kDenomSkip = 1e-12;  // |D| < 1e-12 terms are skipped
                                      // (reference src/mp2/cholesky_rmp2.cc:139)

__host__ __device__ inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t round_up(int64_t a, int64_t b) { return cdiv(a, b) * b; }

// ---------------------------------------------------------------------------
// Neumaier-compensated FP64 accumulation
// ---------------------------------------------------------------------------
struct KSum {
    double s, c;
    __device__ __forceinline__ void init() { s = 0.0; c = 0.0; }
    __device__ __forceinline__ void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

// warp reduction of a compensated sum: (s, c) pairs are combined by TwoSum of
// the heads and plain addition of the tails
__device__ __forceinline__ void warp_reduce_ksum(KSum& k) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        double os = __shfl_xor_sync(0xffffffffu, k.s, off);
        double oc = __shfl_xor_sync(0xffffffffu, k.c, off);
        k.add(os);
        k.c += oc;
    }
}

// ---------------------------------------------------------------------------
// cp.async (Ampere+ asynchronous global->shared copies)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte copy; src_bytes < 16 zero-fills the tail (src_bytes == 0 -> zeros)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)),
                 "l"(gmem), "r"(src_bytes));
}
// 8-byte copy with zero fill
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(smem)),
                 "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---------------------------------------------------------------------------
// DMMA: D(8x8) += A(8x4, row) * B(4x8, col), FP64.
// Fragments per lane l:  a = A[l/4][l%4], b = B[l%4][l/4],
// c0 = C[l/4][2*(l%4)], c1 = C[l/4][2*(l%4)+1].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
    asm volatile(
        "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

}  // namespace mshqc_cd
