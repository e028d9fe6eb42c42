// Batched FP64 GEMM on the FP64 tensor pipe (DMMA m8n8k4), sm_100a.
//
//   C(m, n) = alpha * sum_k A(m, k) B(k, n) + beta * C(m, n)   per batch b
//
// A(m,k) lives at A + b*sA + (A_K ? m*lda + k : k*lda + m)   (A_K: K contiguous)
// B(k,n) lives at B + b*sB + (B_K ? n*ldb + k : k*ldb + n)   (B_K: K contiguous)
// C(m,n) lives at C + b*sC + m*ldc + n
//
// 64x64 CTA tile, K step 16, 4 warps (2x2, 32x32 per warp), two-stage
// cp.async pipeline.  Shared tiles keep the global orientation; the padded
// strides (20 for [row][k], 68 for [k][row]) make the 8-byte fragment reads
// of each half warp hit 16 distinct bank pairs.
#pragma once

#include "cd_common.cuh"

namespace mshqc_cd {

struct GemmF64Args {
    int M, N, K, batch;
    const double* A;
    int64_t lda, sA;
    const double* B;
    int64_t ldb, sB;
    double* C;
    int64_t ldc, sC;
    double alpha, beta;
};

namespace gemm_detail {
constexpr int BM = 64, BN = 64, BK = 16;
constexpr int SK = BK + 4;      // stride of a [row][k] tile
constexpr int SR = BM + 4;      // stride of a [k][row] tile
constexpr int TILE = 64 * SK;   // doubles per operand per stage (>= 16 * SR)
static_assert(TILE >= BK * SR, "tile buffer too small");

// Load one operand tile (rows r0.., k0..) into shared memory.
//   KC = true : element (r, k) at base + r*ld + k  -> smem [r][k] (stride SK)
//   KC = false: element (r, k) at base + k*ld + r  -> smem [k][r] (stride SR)
template <bool KC, int VEC>
__device__ __forceinline__ void load_tile(double* sm, const double* base, int64_t ld,
                                          int r0, int nrows, int k0, int K, int tid) {
    if constexpr (KC) {
        constexpr int CPR = BK / VEC;  // chunks per row
        constexpr int NCH = 64 * CPR;
#pragma unroll
        for (int c = tid; c < NCH; c += 128) {
            int r = c / CPR, kc = (c % CPR) * VEC;
            int gr = r0 + r, gk = k0 + kc;
            int nv = (gr < nrows) ? max(0, min(VEC, K - gk)) : 0;
            const double* src = nv > 0 ? base + (int64_t)gr * ld + gk : base;
            if constexpr (VEC == 2)
                cp_async16(sm + r * SK + kc, src, nv * 8);
            else
                cp_async8(sm + r * SK + kc, src, nv * 8);
        }
    } else {
        constexpr int CPR = 64 / VEC;
        constexpr int NCH = BK * CPR;
#pragma unroll
        for (int c = tid; c < NCH; c += 128) {
            int k = c / CPR, rc = (c % CPR) * VEC;
            int gr = r0 + rc, gk = k0 + k;
            int nv = (gk < K) ? max(0, min(VEC, nrows - gr)) : 0;
            const double* src = nv > 0 ? base + (int64_t)gk * ld + gr : base;
            if constexpr (VEC == 2)
                cp_async16(sm + k * SR + rc, src, nv * 8);
            else
                cp_async8(sm + k * SR + rc, src, nv * 8);
        }
    }
}

template <bool KC>
__device__ __forceinline__ double frag(const double* sm, int r, int k) {
    return KC ? sm[r * SK + k] : sm[k * SR + r];
}
}  // namespace gemm_detail

template <bool A_K, bool B_K, int VEC>
__global__ void __launch_bounds__(128) gemm_f64_kernel(GemmF64Args p) {
    using namespace gemm_detail;
    __shared__ __align__(16) double smA[2][TILE];
    __shared__ __align__(16) double smB[2][TILE];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int64_t b = blockIdx.z;
    const double* A = p.A + b * p.sA;
    const double* B = p.B + b * p.sB;
    double* C = p.C + b * p.sC;

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int nk = (p.K + BK - 1) / BK;
    load_tile<A_K, VEC>(smA[0], A, p.lda, m0, p.M, 0, p.K, tid);
    load_tile<B_K, VEC>(smB[0], B, p.ldb, n0, p.N, 0, p.K, tid);
    cp_async_commit();

    for (int kt = 0; kt < nk; ++kt) {
        const int s = kt & 1;
        if (kt + 1 < nk) {
            load_tile<A_K, VEC>(smA[s ^ 1], A, p.lda, m0, p.M, (kt + 1) * BK, p.K, tid);
            load_tile<B_K, VEC>(smB[s ^ 1], B, p.ldb, n0, p.N, (kt + 1) * BK, p.K, tid);
        }
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const double* sa = smA[s];
        const double* sb = smB[s];
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
                af[i] = frag<A_K>(sa, wm * 32 + i * 8 + (lane >> 2), kk + (lane & 3));
#pragma unroll
            for (int j = 0; j < 4; ++j)
                bf[j] = frag<B_K>(sb, wn * 32 + j * 8 + (lane >> 2), kk + (lane & 3));
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + wm * 32 + i * 8 + (lane >> 2);
        if (m >= p.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int n = n0 + wn * 32 + j * 8 + 2 * (lane & 3) + e;
                if (n >= p.N) continue;
                double* cp = C + (int64_t)m * p.ldc + n;
                double v = p.alpha * acc[i][j][e];
                if (p.beta != 0.0) v += p.beta * (*cp);
                *cp = v;
            }
        }
    }
}

// Host launcher: picks 16-byte copies when every operand row is 16-byte aligned.
inline cudaError_t gemm_f64(const GemmF64Args& a, bool a_k, bool b_k, cudaStream_t st) {
    if (a.M <= 0 || a.N <= 0 || a.batch <= 0) return cudaSuccess;
    dim3 grid((unsigned)cdiv(a.N, 64), (unsigned)cdiv(a.M, 64), (unsigned)a.batch);
    auto al16 = [](const void* ptr, int64_t ld, int64_t s) {
        return (reinterpret_cast<uintptr_t>(ptr) % 16 == 0) && (ld % 2 == 0) && (s % 2 == 0);
    };
    const bool v16 = al16(a.A, a.lda, a.sA) && al16(a.B, a.ldb, a.sB);
#define MSHQC_GEMM_LAUNCH(AK, BK_)                                                   \
    do {                                                                             \
        if (v16)                                                                     \
            gemm_f64_kernel<AK, BK_, 2><<<grid, 128, 0, st>>>(a);                    \
        else                                                                         \
            gemm_f64_kernel<AK, BK_, 1><<<grid, 128, 0, st>>>(a);                    \
    } while (0)
    if (a_k && b_k)
        MSHQC_GEMM_LAUNCH(true, true);
    else if (a_k && !b_k)
        MSHQC_GEMM_LAUNCH(true, false);
    else if (!a_k && b_k)
        MSHQC_GEMM_LAUNCH(false, true);
    else
        MSHQC_GEMM_LAUNCH(false, false);
#undef MSHQC_GEMM_LAUNCH
    return cudaGetLastError();
}

}  // namespace mshqc_cd
