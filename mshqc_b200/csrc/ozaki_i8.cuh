// FP64 matrix products on the 8-bit integer tensor cores (tcgen05 kind::i8)
// by slicing, after Ozaki, Ogita, Oishi and Rump (error-free splitting of
// floating-point matrix products) in the integer form of Ootomo, Ozaki and
// Yokota ("DGEMM on integer matrix multiplication unit", 2024).
//
// Every row r of an operand is scaled by its own power of two 2^e_r with
// max_k |x_rk| < 2^e_r (frexp of the row maximum), rounded to the nearest
// multiple of 2^{e_r - 7S} (an integer m with |m| <= 2^{7S} - 1, so the
// representation error is at most 2^{e_r - 7S - 1} and unbiased) and the
// magnitude of m is cut into S base-128 digits carrying the sign of m:
//   x ~ 2^e_r sum_{s=0}^{S-1} d_s 2^{-7(s+1)},  d_s in [-127, 127].
// A row x times a row y is then
//   2^{e_x + e_y} sum_{w=0}^{S-1} 2^{-7(w+2)} sum_{s+t=w} (d^x_s . d^y_t),
// keeping the S(S+1)/2 slice pairs with s + t < S.  Each slice product is an
// exact 32-bit integer tensor-core accumulation (|sum| <= S 127^2 K < 2^31
// for K <= 26624); the epilogue combines the S weighted sums exactly in 64-bit
// integers and rounds once to FP64.
// With S = 5 the error per term is below about 2^-32 (2^e_x 2^e_y): far
// below the fixed-point splitting that follows on the mixed path, which is
// the only path that uses these products (the FP64 path keeps FP64 FMAs).
//
// Operand storage (per batch, per slice): rows padded to the tile, K padded
// to 32, the UMMA core-matrix K-major blocked layout in bytes
//   (k / 32) * Rp * 32 + ((r / 8) * 2 + (k % 32) / 16) * 128 + (r % 8) * 16 + k % 16
// so the 32-wide K chunk of a 128-row (96-row) tile is one 4 KB (3 KB) copy.
#pragma once

#include <algorithm>

#include "cd_common.cuh"
#include "pair_energy_tc.cuh"
#include "sm100_ptx.cuh"

namespace mshqc_cd {

namespace ozaki {
constexpr int S = 5;                       // slices per operand
constexpr int BM = 128, BN = 96, KB = 32;  // tile rows (A), tile rows (B), K bytes per chunk
constexpr int STAGES = 5;
constexpr uint32_t SLAB_A = BM * KB;       // 4 KB
constexpr uint32_t SLAB_B = BN * KB;       // 3 KB
constexpr uint32_t OFF_B = S * SLAB_A;
constexpr uint32_t STAGE_BYTES = S * (SLAB_A + SLAB_B);   // 35 KB
constexpr uint32_t SMEM_DATA = STAGES * STAGE_BYTES;      // 175 KB
constexpr int STG_LD = 17;                                // epilogue staging row (doubles)
constexpr size_t SMEM_BYTES = SMEM_DATA + 1024 + 256 + 4 * 32 * STG_LD * sizeof(double);
constexpr uint32_t TMEM_COLS = 512;        // S accumulators of BN columns
constexpr uint64_t kWaitLimitNs = 2000000000ull;
constexpr long long kMaxK = 26624;         // S * 127^2 * K < 2^31
static_assert(S * BN <= (int)TMEM_COLS, "accumulators exceed TMEM");
static_assert((long long)S * 127 * 127 * kMaxK < 2147483648LL, "int32 accumulation not exact");

// MMAs of A slice s: its N = (S - s) BN columns in mma_parts(s) equal parts
// of mma_n(s) <= 256 columns (a multiple of 16, and of 8 rows of the B layout)
__host__ __device__ constexpr int mma_parts(int s) { return ((S - s) * BN + 255) / 256; }
__host__ __device__ constexpr int mma_n(int s) { return (S - s) * BN / mma_parts(s); }
constexpr bool mma_split_ok() {
    for (int s = 0; s < S; ++s)
        if (mma_n(s) * mma_parts(s) != (S - s) * BN || mma_n(s) % 16 != 0 || mma_n(s) > 256) return false;
    return true;
}
static_assert(mma_split_ok(), "MMA column split");

inline long long padded_rows(long long rows, int tile) { return (rows + tile - 1) / tile * tile; }
inline long long padded_k(long long k) { return (k + KB - 1) / KB * KB; }
// bytes of one sliced operand (all slices, one batch)
inline size_t operand_bytes(long long Rp, long long Kp) { return (size_t)S * (size_t)Rp * (size_t)Kp; }
}  // namespace ozaki

// Slices of the rows of row-major FP64 matrices (batch b: rows r < R at
// src + b * src_batch + r * ld, K elements each).  One warp per group of 8
// padded rows: lane = (chunk parity, half, row) so that each store of a
// slice is 256 contiguous bytes per 16 lanes.  dst: [batch][slice][Kp x Rp
// bytes]; e: [batch][Rp] row exponents (0 for zero or padding rows).
static __global__ void ozaki_slice_kernel(const double* __restrict__ src, long long ld, long long src_batch,
                                          long long R, long long K, long long Rp, long long Kp, int batch,
                                          int8_t* __restrict__ dst, int* __restrict__ e) {
    using namespace ozaki;
    const long long groups = Rp / 8 * batch;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    const int lane = threadIdx.x & 31;
    const int rr = lane & 7;
    const long long nkc = Kp / KB;
    for (long long gw = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); gw < groups;
         gw += nwarps) {
        const long long b = gw / (Rp / 8), r0 = gw % (Rp / 8) * 8, r = r0 + rr;
        const bool live = r < R;
        const double* row = src + b * src_batch + (live ? r : 0) * ld;
        // row maxima: lanes with equal lane % 8 share a row
        double mx = 0.0;
        if (live)
            for (long long k = lane >> 3; k < K; k += 4) mx = fmax(mx, fabs(row[k]));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
        // |x| < 2^ex; rows below 2^-900 (none in practice) are sliced as zero
        int ex = 0;
        const bool keep = mx >= 0x1p-900;
        if (keep) frexp(mx, &ex);
        if (lane < 8) e[b * Rp + r] = ex;
        const double to_fixed = pow2d(7 * S - ex);
        constexpr long long kMaxFixed = (1LL << (7 * S)) - 1;
        int8_t* out = dst + b * (long long)S * Kp * Rp + (r0 / 8) * 256 + (lane & 15) * 16;
        const int half = (lane >> 3) & 1;
        for (long long kc2 = 0; kc2 < nkc; kc2 += 2) {
            const long long kc = kc2 + (lane >> 4);
            if (kc >= nkc) continue;
            const long long k0 = kc * KB + half * 16;
            uint32_t word[S][4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
#pragma unroll
                for (int s = 0; s < S; ++s) word[s][q] = 0u;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const long long k = k0 + q * 4 + c;
                    // |x| 2^(7S - ex) < 2^(7S): exact scaling, one rounding
                    const double xs = (live && keep && k < K) ? row[k] * to_fixed : 0.0;
                    const long long m = __double2ll_rn(xs);
                    const bool neg = m < 0;
                    const unsigned long long am = (unsigned long long)min(neg ? -m : m, kMaxFixed);
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        const uint32_t d = (uint32_t)(am >> (7 * (S - 1 - s))) & 127u;
                        word[s][q] |= ((neg ? 0u - d : d) & 0xFFu) << (8 * c);
                    }
                }
            }
#pragma unroll
            for (int s = 0; s < S; ++s)
                *reinterpret_cast<uint4*>(out + (long long)s * Kp * Rp + kc * Rp * KB) =
                    make_uint4(word[s][0], word[s][1], word[s][2], word[s][3]);
        }
    }
}

// Slices of the rows of matrices stored with the rows contiguous and K
// strided (batch b: element (r, k) at src + b * src_batch + k * ld + r), in
// three passes: row maxima over K splits (atomicMax of the frexp exponent
// into e, which starts at kNoExponent), exponents of empty or tiny rows set
// to 0, then one thread per (row, 16-wide K group) writing the S digits.
namespace ozaki {
constexpr int kNoExponent = (int)0x80808080;   // byte pattern 0x80 (memset)
constexpr int kTinyExponent = -890;            // rows below 2^-890 are sliced as zero
constexpr int kRowmaxSpan = 512;               // K elements per row-maximum thread
}  // namespace ozaki

static __global__ void __launch_bounds__(256) ozaki_rowmax_t_kernel(const double* __restrict__ src, long long ld,
                                                                    long long src_batch, long long R, long long K,
                                                                    long long Rp, int* __restrict__ e) {
    using namespace ozaki;
    const long long r = blockIdx.x * 256LL + threadIdx.x;
    const long long b = blockIdx.z;
    if (r >= R) return;
    const long long k0 = (long long)blockIdx.y * kRowmaxSpan, k1 = std::min<long long>(K, k0 + kRowmaxSpan);
    const double* col = src + b * src_batch + r;
    double mx = 0.0;
    for (long long k = k0; k < k1; ++k) mx = fmax(mx, fabs(col[k * ld]));
    if (mx > 0.0) {
        int ex = 0;
        frexp(mx, &ex);
        atomicMax(e + b * Rp + r, ex);
    }
}

static __global__ void ozaki_exp_fix_kernel(int* __restrict__ e, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n && e[i] < ozaki::kTinyExponent) e[i] = 0;
}

// grid (Rp / 32, ceil(Kp / 128), batch), 256 threads: lane -> row, warp -> 16-wide K group
static __global__ void __launch_bounds__(256) ozaki_slice_t_kernel(const double* __restrict__ src, long long ld,
                                                                   long long src_batch, long long R, long long K,
                                                                   long long Rp, long long Kp,
                                                                   const int* __restrict__ e,
                                                                   int8_t* __restrict__ dst) {
    using namespace ozaki;
    const int lane = threadIdx.x & 31;
    const long long r = blockIdx.x * 32LL + lane;
    const long long k0 = ((long long)blockIdx.y * 8 + (threadIdx.x >> 5)) * 16;
    const long long b = blockIdx.z;
    if (k0 >= Kp) return;
    const bool live = r < R;
    const int ex = e[b * Rp + r];
    const double to_fixed = pow2d(7 * S - ex);
    constexpr long long kMaxFixed = (1LL << (7 * S)) - 1;
    const double* col = src + b * src_batch + r;
    uint32_t word[S][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int s = 0; s < S; ++s) word[s][q] = 0u;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const long long k = k0 + q * 4 + c;
            const double xs = (live && k < K) ? col[k * ld] * to_fixed : 0.0;
            const long long m = __double2ll_rn(xs);
            const bool neg = m < 0;
            const unsigned long long am = (unsigned long long)min(neg ? -m : m, kMaxFixed);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const uint32_t d = (uint32_t)(am >> (7 * (S - 1 - s))) & 127u;
                word[s][q] |= ((neg ? 0u - d : d) & 0xFFu) << (8 * c);
            }
        }
    }
    int8_t* out = dst + b * (long long)S * Kp * Rp + (k0 >> 5) * Rp * KB +
                  (((r >> 3) * 2 + ((k0 & 31) >> 4)) << 7) + ((r & 7) << 4);
#pragma unroll
    for (int s = 0; s < S; ++s)
        *reinterpret_cast<uint4*>(out + (long long)s * Kp * Rp) =
            make_uint4(word[s][0], word[s][1], word[s][2], word[s][3]);
}

struct OzakiArgs {
    const int8_t* A; long long a_batch; long long RpA; const int* eA; long long ea_batch;
    const int8_t* B; long long b_batch; long long RpB; const int* eB; long long eb_batch;
    long long Kp;              // padded K (multiple of 32)
    int M, N;                  // valid output rows and columns
    int nmb, nnb, batch;       // row blocks (128), column blocks (96), batches
    double* C; long long ldc, c_batch;
    double alpha, beta;
    int* err;
};

// C = alpha * A B^T + beta * C per batch (A: M x K rows, B: N x K rows, both
// sliced).  Warp 0 producer (bulk copies of the S slices of a 32-wide K chunk
// of both tiles), warp 1 MMA issuer and TMEM owner (the S(S+1)/2 slice
// products of a chunk as 8 MMAs into S accumulators), warps 2..5 epilogue
// (exact 64-bit combination, one rounding to FP64, staged through shared
// memory for row-contiguous stores).  Units run row block
// fastest so that concurrent CTAs share the B tile.  Waits are bounded.
static __global__ void __launch_bounds__(192, 1) ozaki_gemm_kernel(OzakiArgs p) {
    using namespace ozaki;
    using namespace sm100;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + SMEM_DATA);
    uint64_t* empty = full + STAGES;
    uint64_t* tmem_full = empty + STAGES;
    uint64_t* tmem_empty = tmem_full + 1;
    uint64_t* drain = tmem_empty + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    double* stg_all = reinterpret_cast<double*>(smem + SMEM_DATA + 256);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(tmem_full, 1);
        mbar_init(tmem_empty, 4);
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const long long per_batch = (long long)p.nmb * p.nnb;
    const long long units = per_batch * p.batch;
    const long long first = blockIdx.x, step = gridDim.x;
    const long long nkc = p.Kp / KB;
    const long long a_slice = p.Kp * p.RpA, b_slice = p.Kp * p.RpB;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t stage = 0, phase = 0, fill_phase = 0, filled = 0;
            for (long long u = first; u < units && !*abort_flag; u += step) {
                const long long b = u / per_batch, rem = u % per_batch;
                const long long nb = rem / p.nmb, mb = rem % p.nmb;
                const int8_t* a0 = p.A + b * p.a_batch + mb * BM * KB;
                const int8_t* b0 = p.B + b * p.b_batch + nb * BN * KB;
                for (long long kc = 0; kc < nkc; ++kc) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 31);
                        *abort_flag = 1;
                        break;
                    }
                    uint8_t* sb = smem + stage * STAGE_BYTES;
                    mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                    const long long ka = kc * p.RpA * KB, kb = kc * p.RpB * KB;
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        bulk_g2s(sb + s * SLAB_A, a0 + s * a_slice + ka, SLAB_A, &full[stage]);
                        bulk_g2s(sb + OFF_B + s * SLAB_B, b0 + s * b_slice + kb, SLAB_B, &full[stage]);
                    }
                    fill_phase = (fill_phase & ~(1u << stage)) | (phase << stage);
                    filled |= 1u << stage;
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
            }
            if (!*abort_flag) {
                for (int s = 0; s < STAGES; ++s) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 35);
                        break;
                    }
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
            } else {
                for (int s = 0; s < STAGES; ++s)
                    if ((filled >> s) & 1u) mbar_wait_bounded(&full[s], (fill_phase >> s) & 1u, kWaitLimitNs);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            uint32_t stage = 0, phase = 0, acc_phase = 0;
            const uint32_t sbase = smem_addr(smem);
            for (long long u = first; u < units && !*abort_flag; u += step) {
                if (!mbar_wait_bounded(tmem_empty, acc_phase ^ 1, kWaitLimitNs)) {
                    atomicExch(p.err, 32);
                    *abort_flag = 1;
                    break;
                }
                acc_phase ^= 1;
                tc_fence_after();
                for (long long kc = 0; kc < nkc; ++kc) {
                    if (!mbar_wait_bounded(&full[stage], phase, kWaitLimitNs)) {
                        atomicExch(p.err, 33);
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sb = sbase + stage * STAGE_BYTES;
                    // A slice s against B slices 0 .. S-1-s in one N = (S - s) BN product
                    // (split in parts of at most 256): B slice t lands in accumulator s + t.
                    // The s = 0 product of the first chunk starts every accumulator.
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        const uint64_t ad = smem_desc_kmajor(sb + s * SLAB_A, 128, 256);
#pragma unroll
                        for (int h = 0; h < mma_parts(s); ++h) {
                            const uint32_t r0 = (uint32_t)(h * mma_n(s));
                            const uint64_t bd = smem_desc_kmajor(sb + OFF_B + r0 * KB, 128, 256);
                            mma_i8(tmem + (uint32_t)(s * BN) + r0, ad, bd, idesc_s8_s32(BM, mma_n(s)),
                                   (kc > 0 || s > 0) ? 1u : 0u);
                        }
                    }
                    mma_commit(&empty[stage]);
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
                if (*abort_flag) break;
                mma_commit(tmem_full);
            }
            mma_commit(drain);
            if (!mbar_wait_bounded(drain, 0, kWaitLimitNs)) atomicExch(p.err, 36);
        }
    } else {
        const int q = warp & 3;
        double* stg = stg_all + (warp - 2) * 32 * STG_LD;
        const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
        const int col = lane & 15, rhalf = lane >> 4;
        uint32_t acc_phase = 0;
        for (long long u = first; u < units; u += step) {
            if (*abort_flag) break;
            const long long b = u / per_batch, rem = u % per_batch;
            const long long nb = rem / p.nmb, mb = rem % p.nmb;
            if (!mbar_wait_bounded(tmem_full, acc_phase, kWaitLimitNs)) {
                atomicExch(p.err, 34);
                *abort_flag = 1;
                break;
            }
            acc_phase ^= 1;
            tc_fence_after();
            const long long m_own = mb * BM + q * 32 + lane;   // this thread's TMEM row
            // T 2^(-7(S+1)) is the scaled product; 2^eA of this row folded in
            const double rs = m_own < p.M ? pow2d(p.eA[b * p.ea_batch + m_own] - 7 * (S + 1)) : 0.0;
            double* Cb = p.C + b * p.c_batch;
            const int* eb = p.eB + b * p.eb_batch;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                uint32_t acc[S][16];
#pragma unroll
                for (int w = 0; w < S; ++w) tmem_ld16(lane_base + (uint32_t)(w * BN + c0), acc[w]);
                tmem_ld_wait();
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    // sum_w acc_w 2^(7(S-1-w)) exactly in 64 bits (|T| < 2^60), one rounding
                    long long T = (long long)(int)acc[0][k];
#pragma unroll
                    for (int w = 1; w < S; ++w) T = T * 128 + (long long)(int)acc[w][k];
                    stg[lane * STG_LD + k] = (double)T * rs;
                }
                __syncwarp();
                // two rows of 16 consecutive columns per store
                const long long n = nb * BN + c0 + col;
                const bool ncol = n < p.N;
                const double cs = ncol ? pow2d(eb[n]) : 0.0;
#pragma unroll 4
                for (int r2 = 0; r2 < 32; r2 += 2) {
                    const int r = r2 + rhalf;
                    const long long m = mb * BM + q * 32 + r;
                    if (ncol && m < p.M) {
                        double* c = Cb + m * p.ldc + n;
                        double out = p.alpha * (stg[r * STG_LD + col] * cs);
                        if (p.beta != 0.0) out = fma(p.beta, *c, out);
                        *c = out;
                    }
                }
                __syncwarp();
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tmem_empty);
        }
    }

    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// ---- host side ---------------------------------------------------------------

// One sliced operand: rows R (padded to Rp), K (padded to Kp), `batch` copies.
struct OzakiOperand {
    int8_t* q = nullptr;
    int* e = nullptr;
    long long R = 0, Rp = 0, K = 0, Kp = 0;
    int batch = 1;
};

inline OzakiOperand ozaki_operand(long long R, long long K, int tile, int batch) {
    OzakiOperand op;
    op.R = R;
    op.Rp = ozaki::padded_rows(R, tile);
    op.K = K;
    op.Kp = ozaki::padded_k(K);
    op.batch = batch;
    return op;
}

inline cudaError_t ozaki_slice(const double* src, long long ld, long long src_batch, const OzakiOperand& op,
                               int num_sms, cudaStream_t st) {
    const long long groups = op.Rp / 8 * op.batch;
    const long long blocks = std::min<long long>((groups + 7) / 8, (long long)num_sms * 16);
    ozaki_slice_kernel<<<(unsigned)std::max<long long>(blocks, 1), 256, 0, st>>>(
        src, ld, src_batch, op.R, op.K, op.Rp, op.Kp, op.batch, op.q, op.e);
    return cudaGetLastError();
}

// Transposed source: element (r, k) of batch b at src + b * src_batch + k * ld + r.
inline cudaError_t ozaki_slice_t(const double* src, long long ld, long long src_batch, const OzakiOperand& op,
                                 cudaStream_t st) {
    using namespace ozaki;
    cudaError_t err = cudaMemsetAsync(op.e, 0x80, sizeof(int) * (size_t)(op.Rp * op.batch), st);
    if (err != cudaSuccess) return err;
    if (op.R > 0 && op.K > 0) {
        dim3 g1((unsigned)((op.R + 255) / 256), (unsigned)((op.K + kRowmaxSpan - 1) / kRowmaxSpan),
                (unsigned)op.batch);
        ozaki_rowmax_t_kernel<<<g1, 256, 0, st>>>(src, ld, src_batch, op.R, op.K, op.Rp, op.e);
        err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    const long long n = op.Rp * op.batch;
    ozaki_exp_fix_kernel<<<(unsigned)std::max<long long>(1, (n + 255) / 256), 256, 0, st>>>(op.e, n);
    err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    dim3 g2((unsigned)(op.Rp / 32), (unsigned)((op.Kp + 127) / 128), (unsigned)op.batch);
    ozaki_slice_t_kernel<<<g2, 256, 0, st>>>(src, ld, src_batch, op.R, op.K, op.Rp, op.Kp, op.e, op.q);
    return cudaGetLastError();
}

// C[b] = alpha * A[b] B[b]^T + beta * C[b] over the batches; a shared operand
// (a_shared / b_shared) is one matrix used by every batch.
inline cudaError_t ozaki_gemm(const OzakiOperand& A, bool a_shared, const OzakiOperand& B, bool b_shared,
                              double* C, long long ldc, long long c_batch, double alpha, double beta, int* err,
                              int num_sms, cudaStream_t st) {
    using namespace ozaki;
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_set[dev]) {
        e = cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_set[dev] = true;
    }
    const int batch = a_shared ? B.batch : A.batch;
    if (A.Kp != B.Kp || A.Kp <= 0 || A.Rp % BM != 0 || B.Rp % BN != 0 || A.K > kMaxK ||
        (!a_shared && !b_shared && A.batch != B.batch) || (a_shared && b_shared && batch != 1))
        return cudaErrorInvalidValue;
    OzakiArgs p{};
    p.A = A.q;  p.a_batch = a_shared ? 0 : (long long)operand_bytes(A.Rp, A.Kp);
    p.RpA = A.Rp;  p.eA = A.e;  p.ea_batch = a_shared ? 0 : A.Rp;
    p.B = B.q;  p.b_batch = b_shared ? 0 : (long long)operand_bytes(B.Rp, B.Kp);
    p.RpB = B.Rp;  p.eB = B.e;  p.eb_batch = b_shared ? 0 : B.Rp;
    p.Kp = A.Kp;
    p.M = (int)A.R;  p.N = (int)B.R;
    p.nmb = (int)(A.Rp / BM);  p.nnb = (int)(B.Rp / BN);  p.batch = batch;
    p.C = C;  p.ldc = ldc;  p.c_batch = c_batch;
    p.alpha = alpha;  p.beta = beta;
    p.err = err;
    const long long units = (long long)p.nmb * p.nnb * p.batch;
    const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>(units, num_sms));
    ozaki_gemm_kernel<<<grid, 192, SMEM_BYTES, st>>>(p);
    return cudaGetLastError();
}

}  // namespace mshqc_cd
