// Gamma GEMM of the MP2 backward on the tensor cores (tcgen05):
//
//   Gamma[(i,a)][Q] = sum_{(j,b)} tt[(i,a)][(j,b)] B[(j,b)][Q]
//
// A operand: the amplitude operand written by amp_elem.cuh (rows (i - i0, a),
// K = (j, b)); B operand: BT, the MO vectors transposed to rows Q, K = (j, b).
// Both are BF16 hi/lo pairs in a row-block-major blocked K-major layout: the
// matrix is cut into blocks of BR rows (128 for A, 256 for B), each block
// stores its 16-wide K chunks one after the other (BR x 16 elements each,
// 8 x 8 core matrices inside), so element (r, k) sits at
//   ((r / BR) * nkc + k / 16) * BR * 16 + ((r % BR) / 8 * 16 + (k % 16) / 8 * 8 + r % 8) * 8 + k % 8
// with nkc the K chunks per block (a_rbs, b_rbs).  Consecutive K steps of a
// tile are contiguous, so one bulk copy moves KS = 2 steps: the copies of a
// 128 x 256 tile are feed-bound at one step per copy (measured: 10.1 ms for a
// launch whose MMAs alone take 7.3 ms; 7.7 ms with two steps per copy).
//
// Tile 128 rows x 256 Q; per 16-wide K step three 128x256x16 MMAs
// (hi.hi + hi.lo + lo.hi).  The K range is cut into chunks of KP steps that
// alternate between two TMEM accumulators; after each chunk the epilogue
// warps add the chunk's FP32 partial into round-to-nearest FP32 register sums,
// so the truncating accumulation of the tensor core only ever spans KP steps.
//
// Warp roles (576 threads): warp 0 producer (bulk copies), warp 1 MMA issuer
// and TMEM owner, warps 2..17 epilogue (TMEM lane quadrant warp % 4, column
// quarter (warp - 2) / 4, 64 accumulators per thread).  Waits are bounded as
// in pair_energy_tc.cuh.
#pragma once

#include <cuda_bf16.h>

#include "cd_common.cuh"
#include "sm100_ptx.cuh"

namespace mshqc_cd {

struct GammaTcArgs {
    const uint16_t* Ahi; const uint16_t* Alo;   // staging (128-row blocks of a_rbs K chunks)
    const uint16_t* Bhi; const uint16_t* Blo;   // BT from the first K chunk used (256-row blocks of b_rbs chunks)
    long long a_rbs, b_rbs;
    int nk;                 // K steps of 16 (even)
    int KP;                 // K steps per promotion chunk
    int nrb, nqb;           // row blocks (of 128) and Q blocks (of 256) to compute
    int VR, v, vp, Mp, i0;  // output mapping R -> (i0 + R / VR, R % VR)
    double* gamma;          // [o][vp][Mp]
    int accumulate;         // 1: gamma += result, 0: gamma = result
    int* err;
    int* pace;              // gridDim.x zeroed progress counters (WavePacer), or null
    int pace_every, pace_slack;
    int group;              // row blocks per tile group (>= 1), see gamma_tile
};

namespace gamma_tc {
constexpr int BM = 128, BN = 256, KC = 16, KS = 2, STAGES = 4, THREADS = 576, EPI_WARPS = 16;
constexpr uint32_t SLAB_A = BM * KC * 2;        // 4 KB per K step
constexpr uint32_t SLAB_B = BN * KC * 2;        // 8 KB per K step
constexpr uint32_t OFF_AH = 0, OFF_AL = KS * SLAB_A, OFF_BH = 2 * KS * SLAB_A, OFF_BL = 2 * KS * SLAB_A + KS * SLAB_B;
constexpr uint32_t STAGE_BYTES = KS * 2 * (SLAB_A + SLAB_B);   // 48 KB: KS steps
constexpr uint32_t SMEM_DATA = STAGES * STAGE_BYTES;           // 192 KB
constexpr size_t SMEM_BYTES = SMEM_DATA + 1024 + 256;
constexpr uint64_t kWaitLimitNs = 2000000000ull;
constexpr uint64_t kPaceLimitNs = 200000ull;   // a pacing wait longer than this turns pacing off
constexpr uint32_t TMEM_COLS = 512;
}  // namespace gamma_tc

// Tile u -> (row block rb, Q block qb).  Tiles come in groups of `group` row
// blocks with all Q blocks, Q-block-major inside a group, so the 148 tiles of
// one wave (consecutive u) span about `group` row blocks and 148 / group Q
// blocks: the operand rows a wave reads, (group * 128 + 148 / group * 256)
// per K step, are fewest near group = 16.  group = 1 is row-block-major.
__device__ __forceinline__ void gamma_tile(const GammaTcArgs& p, long long u, long long& rb, long long& qb) {
    const long long G = p.group, per = G * p.nqb, grp = u / per;
    const long long g0 = grp * G, gsz = min((long long)p.nrb - g0, G);
    const long long w = u - grp * per;
    qb = w / gsz;
    rb = g0 + w % gsz;
}

__global__ void __launch_bounds__(576, 1) gamma_tc_kernel(GammaTcArgs p) {
    using namespace gamma_tc;
    using namespace sm100;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + SMEM_DATA);
    uint64_t* empty = full + STAGES;
    uint64_t* tfull = empty + STAGES;      // [2]
    uint64_t* tempty = tfull + 2;          // [2]
    uint64_t* drain = tempty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI_WARPS);
        }
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

    const long long units = (long long)p.nrb * p.nqb;
    const long long first = blockIdx.x, step = gridDim.x;
    const int nchunks = (p.nk + p.KP - 1) / p.KP;

    if (warp == 0) {
        // producer: lane 0 issues the copies, the whole warp paces
        WavePacer pacer;
        pacer.init(p.pace, (int)gridDim.x, p.pace_every, p.pace_slack);
        uint32_t stage = 0, phase = 0;
        uint32_t fill_phase = 0, filled = 0;   // bit s: parity / presence of stage s's last fill
        bool stop = false;
        for (long long u = first; u < units && !stop; u += step) {
            long long rb, qb;
            gamma_tile(p, u, rb, qb);
            const size_t ra0 = (size_t)rb * p.a_rbs * (BM * 16), rq0 = (size_t)qb * p.b_rbs * (BN * 16);
            for (int kq = 0; kq < p.nk; kq += KS) {
                pacer.step(lane, kPaceLimitNs);
                int ok = 1;
                if (lane == 0) {
                    if (*abort_flag) {
                        ok = 0;
                    } else if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 11);
                        *abort_flag = 1;
                        ok = 0;
                    } else {
                        uint8_t* sb = smem + stage * STAGE_BYTES;
                        mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                        const size_t ka = ra0 + (size_t)kq * (BM * 16), kb = rq0 + (size_t)kq * (BN * 16);
                        bulk_g2s(sb + OFF_AH, p.Ahi + ka, KS * SLAB_A, &full[stage]);
                        bulk_g2s(sb + OFF_AL, p.Alo + ka, KS * SLAB_A, &full[stage]);
                        bulk_g2s(sb + OFF_BH, p.Bhi + kb, KS * SLAB_B, &full[stage]);
                        bulk_g2s(sb + OFF_BL, p.Blo + kb, KS * SLAB_B, &full[stage]);
                    }
                }
                if (!__shfl_sync(0xffffffffu, ok, 0)) {
                    stop = true;
                    break;
                }
                fill_phase = (fill_phase & ~(1u << stage)) | (phase << stage);
                filled |= 1u << stage;
                if (++stage == STAGES) { stage = 0; phase ^= 1; }
            }
        }
        pacer.finish(lane);
        if (lane == 0) {
            if (!*abort_flag) {
                for (int s = 0; s < STAGES; ++s) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 15);
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
            constexpr uint32_t IDESC = idesc_bf16_f32(BM, BN);
            uint32_t stage = 0, phase = 0;
            uint32_t chunk_ctr = 0;      // global chunk counter: buffer = ctr & 1
            const uint32_t sbase = smem_addr(smem);
            for (long long u = first; u < units && !*abort_flag; u += step) {
                int kq = 0;
                for (int c = 0; c < nchunks && !*abort_flag; ++c, ++chunk_ctr) {
                    const uint32_t buf = chunk_ctr & 1, use = chunk_ctr >> 1;
                    if (!mbar_wait_bounded(&tempty[buf], (use & 1) ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 12);
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem + buf * BN;
                    const int kend = min(p.nk, kq + p.KP);
                    for (int ks = 0; kq < kend; kq += KS, ks += KS) {
                        if (!mbar_wait_bounded(&full[stage], phase, kWaitLimitNs)) {
                            atomicExch(p.err, 13);
                            *abort_flag = 1;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t sb = sbase + stage * STAGE_BYTES;
#pragma unroll
                        for (int j = 0; j < KS; ++j) {
                            const uint64_t ah = smem_desc_kmajor(sb + OFF_AH + j * SLAB_A, 128, 256);
                            const uint64_t al = smem_desc_kmajor(sb + OFF_AL + j * SLAB_A, 128, 256);
                            const uint64_t bh = smem_desc_kmajor(sb + OFF_BH + j * SLAB_B, 128, 256);
                            const uint64_t bl = smem_desc_kmajor(sb + OFF_BL + j * SLAB_B, 128, 256);
                            mma_f16(d, ah, bh, IDESC, (ks + j) > 0 ? 1u : 0u);
                            mma_f16(d, ah, bl, IDESC, 1u);
                            mma_f16(d, al, bh, IDESC, 1u);
                        }
                        mma_commit(&empty[stage]);
                        if (++stage == STAGES) { stage = 0; phase ^= 1; }
                    }
                    if (*abort_flag) break;
                    mma_commit(&tfull[buf]);
                }
            }
            mma_commit(drain);
            if (!mbar_wait_bounded(drain, 0, kWaitLimitNs)) atomicExch(p.err, 16);
        }
    } else {
        const int q = warp & 3, part = (warp - 2) >> 2;
        const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16) + part * 64;
        uint32_t chunk_ctr = 0;
        for (long long u = first; u < units; u += step) {
            if (*abort_flag) break;
            float acc[64];
#pragma unroll
            for (int c = 0; c < 64; ++c) acc[c] = 0.0f;
            bool ok = true;
            for (int c = 0; c < nchunks; ++c, ++chunk_ctr) {
                const uint32_t buf = chunk_ctr & 1, use = chunk_ctr >> 1;
                if (!mbar_wait_bounded(&tfull[buf], use & 1, kWaitLimitNs)) {
                    atomicExch(p.err, 14);
                    *abort_flag = 1;
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (int c0 = 0; c0 < 64; c0 += 16) {
                    uint32_t r[16];
                    tmem_ld16(lane_base + buf * BN + c0, r);
                    tmem_ld_wait();
#pragma unroll
                    for (int k = 0; k < 16; ++k) acc[c0 + k] += __uint_as_float(r[k]);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[buf]);
            }
            if (!ok) break;
            // write this thread's row of the tile
            long long rb, qb;
            gamma_tile(p, u, rb, qb);
            const long long R = rb * BM + q * 32 + lane;
            const int i = p.i0 + (int)(R / p.VR), a = (int)(R % p.VR);
            if (a < p.v) {
                // Mp and q0 are multiples of 8 (16-byte aligned blocks of 8)
                const int q0 = (int)(qb * BN) + part * 64;
                double* dst = p.gamma + ((long long)i * p.vp + a) * p.Mp + q0;
#pragma unroll
                for (int c = 0; c < 64; c += 8)
                    if (q0 + c < p.Mp) f32x8_to_f64(dst + c, &acc[c], p.accumulate != 0);
            }
        }
    }

    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

// MO vectors B[j][b][Q] (FP64, [o][vp][Mp]) -> BT hi/lo BF16 with rows Q
// (RQ rows, a multiple of 256), K = (j, b) with b padded to VR; zeros outside
// b < v, Q < M.  Layout: 256-row blocks of o * VR / 16 K chunks (the B
// operand layout of gamma_tc_kernel).
static __global__ void bt_split_kernel(const double* __restrict__ B, int64_t vp, int64_t Mp, int v, int M,
                                       int64_t o, int64_t VR, int64_t RQ, uint16_t* __restrict__ hi,
                                       uint16_t* __restrict__ lo) {
    // one thread = one core-matrix row: 8 consecutive k of one Q
    const int64_t nkc = o * VR / 16;
    const int64_t total = nkc * RQ * 2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t & 7;
        const int64_t kk = (t >> 3) & 1;
        const int64_t rest = t >> 4;                  // kc * (RQ/8) + g
        const int64_t g = rest % (RQ / 8), kc = rest / (RQ / 8);
        const int64_t Q = g * 8 + r;
        const int64_t k0 = kc * 16 + kk * 8;
        uint16_t h[8], l[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int64_t k = k0 + e, j = k / VR, b = k % VR;
            double x = 0.0;
            if (b < v && Q < M) x = B[(j * vp + b) * Mp + Q];
            const __nv_bfloat16 bh = __double2bfloat16(x);
            const __nv_bfloat16 bl = __double2bfloat16(x - (double)__bfloat162float(bh));
            h[e] = __bfloat16_as_ushort(bh);
            l[e] = __bfloat16_as_ushort(bl);
        }
        const int64_t off = ((g >> 5) * nkc + kc) * 4096 + ((g & 31) * 16 + kk * 8 + r) * 8;
        uint4 vh, vl;
        vh.x = h[0] | (uint32_t(h[1]) << 16); vh.y = h[2] | (uint32_t(h[3]) << 16);
        vh.z = h[4] | (uint32_t(h[5]) << 16); vh.w = h[6] | (uint32_t(h[7]) << 16);
        vl.x = l[0] | (uint32_t(l[1]) << 16); vl.y = l[2] | (uint32_t(l[3]) << 16);
        vl.z = l[4] | (uint32_t(l[5]) << 16); vl.w = l[6] | (uint32_t(l[7]) << 16);
        *reinterpret_cast<uint4*>(hi + off) = vh;
        *reinterpret_cast<uint4*>(lo + off) = vl;
    }
}

}  // namespace mshqc_cd
