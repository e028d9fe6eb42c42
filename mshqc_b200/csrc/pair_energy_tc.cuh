// Fused pair-energy kernel on the 5th-generation tensor cores (tcgen05), exact
// fixed-point accumulation (split_bf16.cuh describes the hi/lo encoding).
//
// Operands are the fixed-point hi/lo of split_bf16.cuh in its pair layout:
// 128-row blocks whose 16-wide Q chunks hold the hi slab (4 KB) and then the
// lo slab (4 KB) of the same rows, chunks one after the other, each slab in
// the canonical K-major no-swizzle UMMA layout.  So one contiguous copy
// brings both halves of an operand for KS = 2 chunks (16 KB), and a chunk's
// [hi; lo] is one 256-row operand.
//
// Work unit = pair (i,j), row block x (128 virtuals a), column block y (128
// virtuals b).  Per Q chunk the MMA thread issues four MMAs into four TMEM
// accumulators (columns):
//   [  0,256) P0hi . [P1hi; P1lo]  (N = 256): T1hh in [0,128), hi*lo' in [128,256)
//   [128,256) += P0lo . P1hi       (N = 128): T1x = hi*lo' + lo*hi'
//   [256,512) the same for P2, P3: T2hh in [256,384), T2x in [384,512)
// RESTRICTED / SAME_SPIN: P0 = X_i[x], P1 = X_j[y], P2 = X_j[x], P3 = X_i[y]
//   ->  T1 = (ia|jb), T2 = (ib|ja) at (a,b);
// OPPOSITE_SPIN: P2 = P0, P3 = Y_j[y+1]  ->  T2 = (ia|jb') of the next block.
// A stage holds the four operands' copies for two chunks (64 KB), three
// stages.  The previous form (one 4 KB copy per slab and chunk, six N=128
// MMAs) was bound by the copy rate: eight copies per chunk.
// All accumulator entries are exact integers, so the epilogue recovers
//   (ia|jb) = u_ia u_jb (T1hh + T1x / 256)
// exactly in FP64, substitutes the exact FP64 (ia|ia) on the diagonal, forms
// FP64 denominators and reduces the unit's energy (weights and formulas of
// pair_energy_f64.cuh) into partial[unit].  (ia|jb) and the amplitudes are
// never written to memory.
//
// Warp roles (192 threads): warp 0 producer (bulk copies), warp 1 MMA issuer
// and TMEM owner, warps 2..5 epilogue (TMEM lane quadrant = warp % 4).
// Every wait is bounded (kWaitLimitNs); on a timeout the kernel records the
// site in *err, drains its own copies and MMAs (again bounded), frees TMEM and
// returns.
#pragma once

#include "cd_common.cuh"
#include "pair_energy_f64.cuh"
#include "sm100_ptx.cuh"
#include "split_bf16.cuh"
#include <cuda_bf16.h>

namespace mshqc_cd {

struct PairTcArgs {
    const uint16_t* Xp;     // fixed-point FP16 bits of spin X, pair layout (split_bf16.cuh)
    const uint16_t* Yp;     // spin Y (== X for RESTRICTED / SAME_SPIN)
    const int* ex; const int* ey;               // row exponents [o][rows]
    const double* diag;                         // exact (ia|ia): [ox][rows_x] (RESTRICTED)
                                                // or sum_Q Xa*Yb [diag_o][rows_x] (OPPOSITE)
    int rows_x, rows_y;     // allocated rows per occupied orbital
    int nqc;                // number of 16-wide Q chunks
    int vx, vy;             // virtual counts
    int diag_o, diag_v;     // extent of the opposite-spin diagonal table
    const double* eox; const double* evx;
    const double* eoy; const double* evy;
    const int2* pairs;      // (i, j)
    const int2* blocks;     // (x, y) in 128-blocks
    int nblocks;
    long long units;        // npairs * nblocks
    double* partial;        // [units]
    double* partial2;       // [units] RESTRICTED opposite-spin part
    int* err;               // err[0]: nonzero after a timeout; err[1]: an accumulator reached 2^24
};

namespace pair_tc {
constexpr int BM = 128;
constexpr int BN = 128;
constexpr int KC = 16;
constexpr int KS = 2;                      // Q chunks per stage
constexpr int STAGES = 3;
constexpr int THREADS = 192;
constexpr uint32_t SLAB = 128 * KC * 2;    // 4096 bytes: 128 rows x one chunk, hi or lo
constexpr uint32_t CHUNK = 2 * SLAB;       // hi and lo of one chunk
constexpr uint32_t PIECE = KS * CHUNK;     // one operand of a stage (16 KB)
constexpr uint32_t STAGE_BYTES = 4 * PIECE;                  // 65536: P0 P1 P2 P3
constexpr uint32_t SMEM_DATA = STAGES * STAGE_BYTES;         // 196608
// after the data: barriers (< 256 B), reduction scratch (64 B at +256),
// per-unit column tables at +512: eps (2 x 128 doubles), column scales
// (2 x 128 doubles)
constexpr uint32_t OFF_AUX = 512;
constexpr size_t SMEM_BYTES = SMEM_DATA + 1024 /*align*/ + OFF_AUX + 4 * 128 * 8;
constexpr uint64_t kWaitLimitNs = 2000000000ull;             // 2 s
constexpr uint32_t TMEM_COLS = 512;
}  // namespace pair_tc

// 2^e as a double (|e| well inside the normal range)
__device__ __forceinline__ double pow2d(int e) {
    return __longlong_as_double((long long)(e + 1023) << 52);
}

template <int MODE>
__global__ void __launch_bounds__(192, 1) pair_energy_tc_kernel(PairTcArgs p) {
    using namespace pair_tc;
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
    double* red = reinterpret_cast<double*>(smem + SMEM_DATA + 256);           // 8 doubles
    double* eb_s = reinterpret_cast<double*>(smem + SMEM_DATA + OFF_AUX);      // 256
    double* cs_s = eb_s + 256;                                                 // 256

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

    const long long first = blockIdx.x, step = gridDim.x;
    const int nk = p.nqc;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            uint32_t stage = 0, phase = 0;
            uint32_t fill_phase = 0, filled = 0;   // bit s: parity / presence of stage s's last fill
#pragma unroll
            for (long long u = first; u < p.units && !*abort_flag; u += step) {
                const int2 ij = p.pairs[u / p.nblocks];
                const int2 xy = p.blocks[u % p.nblocks];
                const size_t a0 = (size_t)xy.x * BM, b0 = (size_t)xy.y * BN;
                // operand bases at Q chunk 0 (the 128 rows from r0 of orbital
                // o); chunk kq adds kq * 4096 elements (hi and lo)
                const size_t nbx = (size_t)p.rows_x / 128, nby = (size_t)p.rows_y / 128, nq = (size_t)p.nqc;
                auto slab_x = [&](size_t o, size_t r0) { return ((o * nbx + r0 / 128) * nq) * 4096; };
                auto slab_y = [&](size_t o, size_t r0) { return ((o * nby + r0 / 128) * nq) * 4096; };
                const uint16_t *s0, *s1, *s2, *s3;
                if (MODE == PAIR_OPPOSITE_SPIN) {
                    s0 = p.Xp + slab_x(ij.x, a0);
                    s1 = p.Yp + slab_y(ij.y, b0);
                    s2 = s0;
                    s3 = p.Yp + slab_y(ij.y, b0 + BN);
                } else {
                    s0 = p.Xp + slab_x(ij.x, a0);
                    s1 = p.Xp + slab_x(ij.y, b0);
                    s2 = p.Xp + slab_x(ij.y, a0);
                    s3 = p.Xp + slab_x(ij.x, b0);
                }
                for (int kq = 0; kq < nk; kq += KS) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 1);
                        *abort_flag = 1;
                        break;
                    }
                    const uint32_t bytes = (uint32_t)min(KS, nk - kq) * CHUNK;
                    uint8_t* sb = smem + stage * STAGE_BYTES;
                    mbar_arrive_expect_tx(&full[stage], (MODE == PAIR_OPPOSITE_SPIN ? 3u : 4u) * bytes);
                    const size_t k = (size_t)kq * 4096;
                    bulk_g2s(sb + 0 * PIECE, s0 + k, bytes, &full[stage]);
                    bulk_g2s(sb + 1 * PIECE, s1 + k, bytes, &full[stage]);
                    if (MODE != PAIR_OPPOSITE_SPIN) bulk_g2s(sb + 2 * PIECE, s2 + k, bytes, &full[stage]);
                    bulk_g2s(sb + 3 * PIECE, s3 + k, bytes, &full[stage]);
                    fill_phase = (fill_phase & ~(1u << stage)) | (phase << stage);
                    filled |= 1u << stage;
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
            }
            if (!*abort_flag) {
                // tail: wait until the MMA warp released every stage, so no
                // commit-arrival on an empty barrier is still pending at exit
                for (int s = 0; s < STAGES; ++s) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 5);
                        break;
                    }
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
            } else {
                // aborted: our own copies in flight must land before the CTA exits
                for (int s = 0; s < STAGES; ++s)
                    if ((filled >> s) & 1u) mbar_wait_bounded(&full[s], (fill_phase >> s) & 1u, kWaitLimitNs);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            constexpr uint32_t IDESC = idesc_f16_f32(BM, BN);          // N = 128
            constexpr uint32_t IDESC2 = idesc_f16_f32(BM, 2 * BN);     // N = 256: [hi; lo]
            uint32_t stage = 0, phase = 0, acc_phase = 0;
            const uint32_t sbase = smem_addr(smem);
            for (long long u = first; u < p.units && !*abort_flag; u += step) {
                // accumulators free? (epilogue of the previous unit done)
                if (!mbar_wait_bounded(tmem_empty, acc_phase ^ 1, kWaitLimitNs)) {
                    atomicExch(p.err, 2);
                    *abort_flag = 1;
                    break;
                }
                acc_phase ^= 1;
                tc_fence_after();
                for (int kq = 0; kq < nk; kq += KS) {
                    if (!mbar_wait_bounded(&full[stage], phase, kWaitLimitNs)) {
                        atomicExch(p.err, 3);
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sb = sbase + stage * STAGE_BYTES;
                    const int nks = min(KS, nk - kq);
                    for (int c = 0; c < nks; ++c) {
                        const uint32_t o0 = sb + 0 * PIECE + c * CHUNK, o1 = sb + 1 * PIECE + c * CHUNK;
                        const uint32_t o2 = (MODE == PAIR_OPPOSITE_SPIN ? sb : sb + 2 * PIECE) + c * CHUNK;
                        const uint32_t o3 = sb + 3 * PIECE + c * CHUNK;
                        // hi at +0, lo at +SLAB; [hi; lo] is the 256-row operand at +0
                        const uint64_t p0h = smem_desc_kmajor(o0, 128, 256), p0l = smem_desc_kmajor(o0 + SLAB, 128, 256);
                        const uint64_t p2h = smem_desc_kmajor(o2, 128, 256), p2l = smem_desc_kmajor(o2 + SLAB, 128, 256);
                        const uint64_t p1 = smem_desc_kmajor(o1, 128, 256), p3 = smem_desc_kmajor(o3, 128, 256);
                        const uint32_t acc = (kq + c) > 0 ? 1u : 0u;
                        mma_f16(tmem + 0, p0h, p1, IDESC2, acc);     // hh | hi*lo'
                        mma_f16(tmem + 128, p0l, p1, IDESC, 1u);     // + lo*hi'
                        mma_f16(tmem + 256, p2h, p3, IDESC2, acc);
                        mma_f16(tmem + 384, p2l, p3, IDESC, 1u);
                    }
                    mma_commit(&empty[stage]);       // frees the stage when these MMAs finish
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
                if (*abort_flag) break;
                mma_commit(tmem_full);                // accumulators ready for the epilogue
            }
            // every MMA this thread issued has finished before TMEM is freed
            mma_commit(drain);
            if (!mbar_wait_bounded(drain, 0, kWaitLimitNs)) atomicExch(p.err, 6);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int q = warp & 3;                       // TMEM lane quadrant of this warp
        const int row = q * 32 + lane;                // a offset within the row block
        const int etid = threadIdx.x - 64;            // 0..127
        uint32_t acc_phase = 0;
        for (long long u = first; u < p.units; u += step) {
            const int2 ij = p.pairs[u / p.nblocks];
            const int2 xy = p.blocks[u % p.nblocks];
            const int i = ij.x, j = ij.y;
            const int a = xy.x * BM + row;
            const int b0 = xy.y * BN;
            // per-unit column tables (eps and scales of T1 / T2 columns)
            for (int c = etid; c < 2 * BN; c += 128) {
                const int half = c / BN, cc = c % BN;
                double eb = 0.0, cs = 0.0;
                if (MODE == PAIR_OPPOSITE_SPIN) {
                    const int b = b0 + half * BN + cc;
                    if (b < p.vy) {
                        eb = p.evy[b];
                        cs = pow2d(p.ey[(size_t)j * p.rows_y + b] - kFixedHiBits);
                    }
                } else {
                    const int b = b0 + cc;
                    if (b < p.vx) {
                        eb = p.evx[b];
                        // T1 columns are rows of X_j, T2 columns rows of X_i
                        cs = pow2d(p.ex[(size_t)(half == 0 ? j : i) * p.rows_x + b] - kFixedHiBits);
                    }
                }
                eb_s[c] = eb;
                cs_s[c] = cs;
            }
            // the four epilogue warps leave together (a named barrier must
            // never wait for a warp that already left the loop)
            if (bar_any(1, 128, *abort_flag != 0)) break;
            const bool got = mbar_wait_bounded(tmem_full, acc_phase, kWaitLimitNs);
            if (bar_any(1, 128, !got)) {
                if (!got) atomicExch(p.err, 4);
                *abort_flag = 1;
                break;
            }
            acc_phase ^= 1;
            tc_fence_after();

            const bool arow = a < p.vx;
            double rs1 = 0.0, rs2 = 0.0, ta = 0.0, dg1 = 0.0, dg2 = 0.0;
            int dcol1 = -1, dcol2 = -1;   // column holding a == b (exact diagonal), if any
            if (arow) {
                if (MODE == PAIR_OPPOSITE_SPIN) {
                    rs1 = rs2 = pow2d(p.ex[(size_t)i * p.rows_x + a] - kFixedHiBits);
                    ta = p.eox[i] + p.eoy[j] - p.evx[a];
                    if (i == j && i < p.diag_o && a < p.diag_v) {
                        const int c1 = a - b0, c2 = a - b0 - BN;
                        if (c1 >= 0 && c1 < BN) { dcol1 = c1; dg1 = p.diag[(size_t)i * p.rows_x + a]; }
                        if (c2 >= 0 && c2 < BN) { dcol2 = c2; dg2 = p.diag[(size_t)i * p.rows_x + a]; }
                    }
                } else {
                    rs1 = pow2d(p.ex[(size_t)i * p.rows_x + a] - kFixedHiBits);
                    rs2 = pow2d(p.ex[(size_t)j * p.rows_x + a] - kFixedHiBits);
                    ta = p.eox[i] + p.eox[j] - p.evx[a];
                    if (MODE == PAIR_RESTRICTED && i == j && a >= b0 && a < b0 + BN) {
                        dcol1 = dcol2 = a - b0;
                        dg1 = dg2 = p.diag[(size_t)i * p.rows_x + a];
                    }
                }
            }
            double s_acc = 0.0, o_acc = 0.0;
            float amax = 0.0f;
            const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
            constexpr int CW = 32;   // columns per TMEM read
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += CW) {
                uint32_t h1[CW], x1[CW], h2[CW], x2[CW];
                tmem_ld<CW>(lane_base + 0 + c0, h1);
                tmem_ld<CW>(lane_base + 128 + c0, x1);
                tmem_ld<CW>(lane_base + 256 + c0, h2);
                tmem_ld<CW>(lane_base + 384 + c0, x2);
                tmem_ld_wait();
                if (!arow) continue;
#pragma unroll
                for (int k = 0; k < CW; ++k) {
                    const int c = c0 + k;
                    amax = fmaxf(amax, fmaxf(fmaxf(fabsf(__uint_as_float(h1[k])), fabsf(__uint_as_float(x1[k]))),
                                             fmaxf(fabsf(__uint_as_float(h2[k])), fabsf(__uint_as_float(x2[k])))));
                    double v1 = fma((double)__uint_as_float(x1[k]), 1.0 / kFixedLoScale,
                                    (double)__uint_as_float(h1[k])) * (rs1 * cs_s[c]);
                    double v2 = fma((double)__uint_as_float(x2[k]), 1.0 / kFixedLoScale,
                                    (double)__uint_as_float(h2[k])) * (rs2 * cs_s[BN + c]);
                    if (c == dcol1) v1 = dg1;
                    if (c == dcol2) v2 = dg2;
                    if (MODE == PAIR_OPPOSITE_SPIN) {
                        if (b0 + c < p.vy) {
                            const double D = ta - eb_s[c];
                            if (fabs(D) >= kDenomSkip) s_acc = fma(v1 * v1, recip_nr(D), s_acc);
                        }
                        if (b0 + BN + c < p.vy) {
                            const double D = ta - eb_s[BN + c];
                            if (fabs(D) >= kDenomSkip) s_acc = fma(v2 * v2, recip_nr(D), s_acc);
                        }
                    } else if (b0 + c < p.vx) {
                        const double D = ta - eb_s[c];
                        if (fabs(D) >= kDenomSkip) {
                            const double rD = recip_nr(D);
                            if (MODE == PAIR_RESTRICTED) {
                                const double sq = fma(v1, v1, v2 * v2);
                                s_acc = fma(fma(-v1, v2, sq), rD, s_acc);
                                o_acc = fma(sq, rD, o_acc);
                            } else {
                                const double g = v1 - v2;
                                s_acc = fma(g * g, rD, s_acc);
                            }
                        }
                    }
                }
            }
            // accumulators consumed: hand TMEM back to the MMA warp
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tmem_empty);
            if (amax >= 16777216.0f) atomicOr(p.err + 1, 1);

            // unit weights (see pair_energy_f64.cuh)
            double tot1 = s_acc, tot2 = 0.0;
            if (MODE != PAIR_OPPOSITE_SPIN) {
                const bool diagblk = (xy.x == xy.y);
                if (MODE == PAIR_RESTRICTED) {
                    const double w = (diagblk ? 1.0 : 2.0) * (i < j ? 2.0 : 1.0);
                    tot1 = w * s_acc;
                    tot2 = 0.5 * w * o_acc;
                } else {
                    tot1 = (diagblk ? 0.5 : 1.0) * s_acc;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                tot1 += __shfl_xor_sync(0xffffffffu, tot1, off);
                tot2 += __shfl_xor_sync(0xffffffffu, tot2, off);
            }
            if (lane == 0) {
                red[q] = tot1;
                red[4 + q] = tot2;
            }
            asm volatile("bar.sync 1, 128;\n" ::: "memory");
            if (etid == 0) {
                p.partial[u] = ((red[0] + red[1]) + (red[2] + red[3]));
                if (MODE == PAIR_RESTRICTED) p.partial2[u] = ((red[4] + red[5]) + (red[6] + red[7]));
            }
        }
    }

    // ---------------------------------------------------------------- teardown
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

}  // namespace mshqc_cd
