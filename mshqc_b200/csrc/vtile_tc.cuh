// Integral tiles of the MP2 backward on the tensor cores (tcgen05):
//
//   S[(i - i0, a)][(j, b)] = (ia|jb) = sum_Q X^Q_ia Y^Q_jb     (FP32)
//
// for the occupied rows i of one block and the columns j of another (or all
// j), every tile computed once;
// X and Y are the MO vectors of one spin (restricted, same spin) or of the
// two spins (opposite spin: X alpha, Y beta).
// Operands are the exact fixed-point hi/lo of split_bf16.cuh in its 256-row
// blocked layout; a stage holds KS = 2 Q steps: the A slab (128 rows) per
// step, the B slab (256 rows) of both steps in one copy (one-step copies
// left the kernel feed-bound: 7.7 ms for a launch whose MMAs take 5.8 ms;
// 5.9 ms with the two-step B copies).  Per 16-wide Q step three 128x256x16 MMAs
// accumulate the hi*hi' and the hi*lo' + lo*hi' integers exactly in two TMEM
// accumulators (columns [0,256) and [256,512)), and the epilogue recovers
//   (ia|jb) = u_ia u_jb (hh + x / 256)
// in FP64, substitutes the exact (ia|ia) for i = j, a = b when X = Y, and
// stores it rounded to FP32 into the row-major staging matrix S (row length
// nbj * VS).  amp_elem.cuh turns S into amplitudes.
//
// Warp roles (192 threads): warp 0 producer, warp 1 MMA issuer and TMEM
// owner, warps 2..5 epilogue.  Waits are bounded as in pair_energy_tc.cuh.
#pragma once

#include "cd_common.cuh"
#include "pair_energy_tc.cuh"
#include "sm100_ptx.cuh"
#include "split_bf16.cuh"

namespace mshqc_cd {

struct VtileArgs {
    const uint16_t* Xhi; const uint16_t* Xlo;   // blocked fixed-point operands (rows i, a)
    const uint16_t* Yhi; const uint16_t* Ylo;   // (columns j, b)
    const int* ex; const int* ey;               // row exponents [o][rows]
    const double* diag;                         // exact (ia|ia) [o][rows_x] when X = Y, else null
    int rows_x, rows_y;     // allocated rows per occupied orbital (operand layouts)
    int nqc;                // 16-wide Q chunks
    int j0, nbj;            // column orbitals j0 .. j0 + nbj - 1
    int vx, vy, VR, i0, nbi;       // VR: staging rows per orbital i (nbx * 128)
    int nbx, nby;           // row blocks (128) per orbital i, column ranges (256) per orbital j
    int VS;                 // staging columns per orbital j (nby * 256)
    float* S;               // staging [nbi * VR][nbj * VS]
    int* err;
    int tri;                // 1: only the pairs ii <= jj of a diagonal block (nbi == nbj)
    int* pace;              // gridDim.x zeroed progress counters (WavePacer), or null
    int pace_every, pace_slack;
};

// Local pair pr -> (ii, jj): row-major over nbi x nbj, or over the upper
// triangle ii <= jj (rows of nbi - ii pairs) when p.tri.
__device__ __forceinline__ void vtile_pair(const VtileArgs& p, long long pr, int& ii, int& jj) {
    if (!p.tri) {
        ii = (int)(pr / p.nbj);
        jj = (int)(pr % p.nbj);
        return;
    }
    int r = (int)pr, i = 0;
    while (r >= p.nbi - i) {
        r -= p.nbi - i;
        ++i;
    }
    ii = i;
    jj = i + r;
}

namespace vtile_tc {
constexpr int BM = 128, BN = 256, KC = 16, KS = 2, STAGES = 4, THREADS = 192;
constexpr uint32_t SLAB_A = BM * KC * 2;     // 4 KB per Q step
constexpr uint32_t SLAB_B = BN * KC * 2;     // 8 KB per Q step
constexpr uint32_t OFF_AH = 0, OFF_AL = KS * SLAB_A, OFF_BH = 2 * KS * SLAB_A, OFF_BL = 2 * KS * SLAB_A + KS * SLAB_B;
constexpr uint32_t STAGE_BYTES = KS * 2 * (SLAB_A + SLAB_B);   // 48 KB
constexpr uint32_t SMEM_DATA = STAGES * STAGE_BYTES;           // 192 KB
constexpr size_t SMEM_BYTES = SMEM_DATA + 1024 + 256 + BN * 8;
constexpr uint64_t kWaitLimitNs = 2000000000ull;
constexpr uint64_t kPaceLimitNs = 200000ull;   // a pacing wait longer than this turns pacing off
constexpr uint32_t TMEM_COLS = 512;
}  // namespace vtile_tc

__global__ void __launch_bounds__(192, 1) vtile_tc_kernel(VtileArgs p) {
    using namespace vtile_tc;
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
    double* cs_s = reinterpret_cast<double*>(smem + SMEM_DATA + 256);   // BN column scales

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

    // unit u -> (ii, j, x, y): pair-major so that concurrent CTAs share slabs
    const long long per_pair = (long long)p.nbx * p.nby;
    const long long npl = p.tri ? (long long)p.nbi * (p.nbi + 1) / 2 : (long long)p.nbi * p.nbj;
    const long long units = npl * per_pair;
    const long long first = blockIdx.x, step = gridDim.x;
    const int nk = p.nqc;

    if (warp == 0) {
        // producer: lane 0 issues the copies, the whole warp paces
        WavePacer pacer;
        pacer.init(p.pace, (int)gridDim.x, p.pace_every, p.pace_slack);
        uint32_t stage = 0, phase = 0, fill_phase = 0, filled = 0;
        bool stop = false;
        for (long long u = first; u < units && !stop; u += step) {
            const long long pr = u / per_pair, bb = u % per_pair;
            int ii, jj;
            vtile_pair(p, pr, ii, jj);
            const int i = p.i0 + ii, j = p.j0 + jj;
            const int x = (int)(bb / p.nby), y = (int)(bb % p.nby);
            // slab bases at Q step 0 (256-row blocks of nqc steps, 4096 elements a step)
            const size_t nq = (size_t)p.nqc;
            const size_t xa = (((size_t)i * (p.rows_x / 256) + x / 2) * nq) * 4096 + (size_t)(x % 2) * 2048;
            const size_t yb = (((size_t)j * (p.rows_y / 256) + y) * nq) * 4096;
            const uint16_t* ah = p.Xhi + xa;
            const uint16_t* al = p.Xlo + xa;
            const uint16_t* bh = p.Yhi + yb;
            const uint16_t* bl = p.Ylo + yb;
            for (int kq = 0; kq < nk; kq += KS) {
                pacer.step(lane, kPaceLimitNs);
                int ok = 1;
                if (lane == 0) {
                    if (*abort_flag) {
                        ok = 0;
                    } else if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 21);
                        *abort_flag = 1;
                        ok = 0;
                    } else {
                        const int nks = min(KS, nk - kq);
                        uint8_t* sb = smem + stage * STAGE_BYTES;
                        mbar_arrive_expect_tx(&full[stage], (uint32_t)nks * 2 * (SLAB_A + SLAB_B));
                        const size_t kk = (size_t)kq * 4096;
                        for (int q2 = 0; q2 < nks; ++q2) {
                            bulk_g2s(sb + OFF_AH + q2 * SLAB_A, ah + kk + q2 * 4096, SLAB_A, &full[stage]);
                            bulk_g2s(sb + OFF_AL + q2 * SLAB_A, al + kk + q2 * 4096, SLAB_A, &full[stage]);
                        }
                        bulk_g2s(sb + OFF_BH, bh + kk, nks * SLAB_B, &full[stage]);
                        bulk_g2s(sb + OFF_BL, bl + kk, nks * SLAB_B, &full[stage]);
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
                        atomicExch(p.err, 25);
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
            constexpr uint32_t IDESC = idesc_f16_f32(BM, BN);
            uint32_t stage = 0, phase = 0, acc_phase = 0;
            const uint32_t sbase = smem_addr(smem);
            for (long long u = first; u < units && !*abort_flag; u += step) {
                if (!mbar_wait_bounded(tmem_empty, acc_phase ^ 1, kWaitLimitNs)) {
                    atomicExch(p.err, 22);
                    *abort_flag = 1;
                    break;
                }
                acc_phase ^= 1;
                tc_fence_after();
                for (int kq = 0; kq < nk; kq += KS) {
                    if (!mbar_wait_bounded(&full[stage], phase, kWaitLimitNs)) {
                        atomicExch(p.err, 23);
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sb = sbase + stage * STAGE_BYTES;
                    const int nks = min(KS, nk - kq);
                    for (int q2 = 0; q2 < nks; ++q2) {
                        const uint64_t ah = smem_desc_kmajor(sb + OFF_AH + q2 * SLAB_A, 128, 256);
                        const uint64_t al = smem_desc_kmajor(sb + OFF_AL + q2 * SLAB_A, 128, 256);
                        const uint64_t bh = smem_desc_kmajor(sb + OFF_BH + q2 * SLAB_B, 128, 256);
                        const uint64_t bl = smem_desc_kmajor(sb + OFF_BL + q2 * SLAB_B, 128, 256);
                        const uint32_t acc = (kq + q2) > 0 ? 1u : 0u;
                        mma_f16(tmem, ah, bh, IDESC, acc);
                        mma_f16(tmem + BN, ah, bl, IDESC, acc);
                        mma_f16(tmem + BN, al, bh, IDESC, 1u);
                    }
                    mma_commit(&empty[stage]);
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
                if (*abort_flag) break;
                mma_commit(tmem_full);
            }
            mma_commit(drain);
            if (!mbar_wait_bounded(drain, 0, kWaitLimitNs)) atomicExch(p.err, 26);
        }
    } else {
        const int q = warp & 3;
        const int row = q * 32 + lane;
        const int etid = threadIdx.x - 64;
        const long long ldS = (long long)p.nbj * p.VS;
        uint32_t acc_phase = 0;
        for (long long u = first; u < units; u += step) {
            const long long pr = u / per_pair, bb = u % per_pair;
            int ii, jj;
            vtile_pair(p, pr, ii, jj);
            const int i = p.i0 + ii, j = p.j0 + jj;
            const int x = (int)(bb / p.nby), y = (int)(bb % p.nby);
            const int a = x * BM + row, b0 = y * BN;
            for (int c = etid; c < BN; c += 128) {
                const int b = b0 + c;
                cs_s[c] = (b < p.vy) ? pow2d(p.ey[(size_t)j * p.rows_y + b] - kFixedHiBits) : 0.0;
            }
            // the four epilogue warps leave together (a named barrier must
            // never wait for a warp that already left the loop)
            if (bar_any(1, 128, *abort_flag != 0)) break;
            const bool got = mbar_wait_bounded(tmem_full, acc_phase, kWaitLimitNs);
            if (bar_any(1, 128, !got)) {
                if (!got) atomicExch(p.err, 24);
                *abort_flag = 1;
                break;
            }
            acc_phase ^= 1;
            tc_fence_after();
            const bool arow = a < p.vx;
            const double rs = arow ? pow2d(p.ex[(size_t)i * p.rows_x + a] - kFixedHiBits) : 0.0;
            const int dcol = (p.diag && arow && i == j && a >= b0 && a < b0 + BN) ? a - b0 : -1;
            const double dg = dcol >= 0 ? p.diag[(size_t)i * p.rows_x + a] : 0.0;
            float* dst = p.S + ((long long)ii * p.VR + a) * ldS + (long long)jj * p.VS + b0;
            const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
            float amax = 0.0f;   // integer accumulators stay exact below 2^24
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                uint32_t h[16], xx[16];
                tmem_ld16(lane_base + c0, h);
                tmem_ld16(lane_base + BN + c0, xx);
                tmem_ld_wait();
                float out[16];
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    amax = fmaxf(amax, fmaxf(fabsf(__uint_as_float(h[k])), fabsf(__uint_as_float(xx[k]))));
                    double V = fma((double)__uint_as_float(xx[k]), 1.0 / kFixedLoScale,
                                   (double)__uint_as_float(h[k])) * (rs * cs_s[c0 + k]);
                    if (c0 + k == dcol) V = dg;
                    out[k] = arow ? (float)V : 0.0f;
                }
                if (a < p.VR) {
                    // streaming stores (evict first): the staging is read once
                    // by the element-wise pass, and must not push the
                    // operands that other CTAs still read out of L2
                    float4* d4 = reinterpret_cast<float4*>(dst + c0);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        __stcs(d4 + k, make_float4(out[4 * k], out[4 * k + 1], out[4 * k + 2], out[4 * k + 3]));
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tmem_empty);
            if (amax >= 16777216.0f) atomicOr(p.err + 1, 1);
            asm volatile("bar.sync 1, 128;\n" ::: "memory");   // cs_s reused by the next unit
        }
    }

    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace mshqc_cd
