// Fused BF16x3 pair-energy kernel on the 5th-generation tensor cores (tcgen05).
//
// Operands: the MO vectors split as B = hi + lo (both BF16), stored in a
// "core-matrix blocked" layout so that every operand slab is one contiguous
// run of bytes and lands in shared memory already in the canonical K-major
// no-swizzle UMMA layout:
//
//   element (i, a, Q) at  (i*nqc + Q/16)*rows*16 + (a/8*16 + (Q%16)/8*8 + a%8)*8 + Q%8
//
// (rows = allocated virtual rows per occupied orbital, a multiple of 128 plus
// one spare block of zeros).  A slab = rows [a0, a0+R) x Q-chunk of 16 =
// R*32 contiguous bytes.
//
// One work unit = pair (i,j), virtual row block x (128 rows of a), column
// range starting at 128-block y (256 columns of b).  Per 16-wide Q step the
// MMA warp issues six 128x256x16 MMAs accumulating in TMEM:
//   T1 (cols 0..255)   += Xhi_i[x] Yhi_j[y]^T + Xhi_i[x] Ylo_j[y]^T + Xlo_i[x] Yhi_j[y]^T
//   T2 (cols 256..511) += (same with slabs P2, P3)
// RESTRICTED / SAME_SPIN: T1 = (ia|jb), T2 = (ib|ja) at the same (a,b);
// OPPOSITE_SPIN: T1, T2 = (ia|jb) for column ranges y and y+2 (blocks of 128).
// The epilogue warps read the accumulators with tcgen05.ld, form the FP64
// denominators and reduce the energy of the unit into partial[unit] (FP64)
// without ever writing (ia|jb) or the amplitudes to memory.  Element weights
// and formulas are those of the FP64 kernel (pair_energy_f64.cuh).
//
// Warp roles (192 threads): warp 0 producer (bulk copies), warp 1 MMA issuer
// and TMEM owner, warps 2..5 epilogue (TMEM lane quadrant = warp % 4).
// Every wait is bounded (kWaitLimitNs); on a timeout the kernel records the
// place in *err, drains its own copies and MMAs (again bounded), frees TMEM and
// returns.
#pragma once

#include "cd_common.cuh"
#include "pair_energy_f64.cuh"
#include "sm100_ptx.cuh"

namespace mshqc_cd {

struct PairTcArgs {
    const uint16_t* Xhi; const uint16_t* Xlo;   // blocked BF16 bits, spin X
    const uint16_t* Yhi; const uint16_t* Ylo;   // spin Y (== X for RESTRICTED / SAME_SPIN)
    int rows_x, rows_y;     // allocated rows per occupied orbital (multiple of 128, + 128 spare)
    int nqc;                // number of 16-wide Q chunks
    int vx, vy;             // virtual counts
    const double* eox; const double* evx;
    const double* eoy; const double* evy;
    const int2* pairs;      // (i, j)
    const int2* blocks;     // (x, y) in 128-blocks
    int nblocks;
    long long units;        // npairs * nblocks
    double* partial;        // [units]
    double* partial2;       // [units] RESTRICTED opposite-spin part
    int* err;               // nonzero after a timeout
};

namespace pair_tc {
constexpr int BM = 128;
constexpr int BN = 256;
constexpr int KC = 16;
constexpr int STAGES = 4;
constexpr int THREADS = 192;
constexpr uint32_t SLAB_A = BM * KC * 2;   // 4096 bytes
constexpr uint32_t SLAB_B = BN * KC * 2;   // 8192 bytes
// stage layout: P0hi P1hi P2hi P3hi P0lo P1lo P2lo P3lo
constexpr uint32_t OFF_P0 = 0, OFF_P1 = SLAB_A, OFF_P2 = SLAB_A + SLAB_B, OFF_P3 = 2 * SLAB_A + SLAB_B;
constexpr uint32_t HALF = 2 * (SLAB_A + SLAB_B);           // 24576
constexpr uint32_t STAGE_BYTES = 2 * HALF;                  // 49152
constexpr uint32_t SMEM_DATA = STAGES * STAGE_BYTES;        // 196608
constexpr size_t SMEM_BYTES = SMEM_DATA + 1024 /*align*/ + 512 /*barriers, eps*/ + BN * 2 * 8;
constexpr uint64_t kWaitLimitNs = 2000000000ull;            // 2 s
constexpr uint32_t TMEM_COLS = 512;
}  // namespace pair_tc

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
    double* red = reinterpret_cast<double*>(smem + SMEM_DATA + 128);        // 2 x 4 warps
    double* eb_s = reinterpret_cast<double*>(smem + SMEM_DATA + 512);       // 2 x 256

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
            uint32_t fill_phase[STAGES];
            bool filled[STAGES];
#pragma unroll
            for (int s = 0; s < STAGES; ++s) { fill_phase[s] = 0; filled[s] = false; }
            for (long long u = first; u < p.units && !*abort_flag; u += step) {
                const int2 ij = p.pairs[u / p.nblocks];
                const int2 xy = p.blocks[u % p.nblocks];
                const size_t rx = p.rows_x, ry = p.rows_y;
                const uint16_t *p0h, *p1h, *p2h, *p3h, *p0l, *p1l, *p2l, *p3l;
                // slab bases at Q-chunk 0; chunk qc adds qc * rows * 16 elements
                const size_t a0 = (size_t)xy.x * BM, b0 = (size_t)xy.y * 128;
                if (MODE == PAIR_OPPOSITE_SPIN) {
                    const size_t oi = (size_t)ij.x * p.nqc * rx * 16, oj = (size_t)ij.y * p.nqc * ry * 16;
                    p0h = p.Xhi + oi + a0 * 16;  p0l = p.Xlo + oi + a0 * 16;
                    p1h = p.Yhi + oj + b0 * 16;  p1l = p.Ylo + oj + b0 * 16;
                    p2h = p0h;                   p2l = p0l;
                    p3h = p.Yhi + oj + (b0 + BN) * 16;  p3l = p.Ylo + oj + (b0 + BN) * 16;
                } else {
                    const size_t oi = (size_t)ij.x * p.nqc * rx * 16, oj = (size_t)ij.y * p.nqc * rx * 16;
                    p0h = p.Xhi + oi + a0 * 16;  p0l = p.Xlo + oi + a0 * 16;
                    p1h = p.Xhi + oj + b0 * 16;  p1l = p.Xlo + oj + b0 * 16;
                    p2h = p.Xhi + oj + a0 * 16;  p2l = p.Xlo + oj + a0 * 16;
                    p3h = p.Xhi + oi + b0 * 16;  p3l = p.Xlo + oi + b0 * 16;
                }
                const size_t cx = rx * 16, cy = (MODE == PAIR_OPPOSITE_SPIN) ? ry * 16 : rx * 16;
                const uint32_t bytes = (MODE == PAIR_OPPOSITE_SPIN) ? 2 * (SLAB_A + 2 * SLAB_B) : STAGE_BYTES;
                for (int kq = 0; kq < nk; ++kq) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 1);
                        *abort_flag = 1;
                        break;
                    }
                    uint8_t* sb = smem + stage * STAGE_BYTES;
                    mbar_arrive_expect_tx(&full[stage], bytes);
                    const size_t qx = (size_t)kq * cx, qy = (size_t)kq * cy;
                    bulk_g2s(sb + OFF_P0, p0h + qx, SLAB_A, &full[stage]);
                    bulk_g2s(sb + HALF + OFF_P0, p0l + qx, SLAB_A, &full[stage]);
                    bulk_g2s(sb + OFF_P1, p1h + qy, SLAB_B, &full[stage]);
                    bulk_g2s(sb + HALF + OFF_P1, p1l + qy, SLAB_B, &full[stage]);
                    if (MODE != PAIR_OPPOSITE_SPIN) {
                        bulk_g2s(sb + OFF_P2, p2h + qy, SLAB_A, &full[stage]);
                        bulk_g2s(sb + HALF + OFF_P2, p2l + qy, SLAB_A, &full[stage]);
                        bulk_g2s(sb + OFF_P3, p3h + qx, SLAB_B, &full[stage]);
                        bulk_g2s(sb + HALF + OFF_P3, p3l + qx, SLAB_B, &full[stage]);
                    } else {
                        bulk_g2s(sb + OFF_P3, p3h + qy, SLAB_B, &full[stage]);
                        bulk_g2s(sb + HALF + OFF_P3, p3l + qy, SLAB_B, &full[stage]);
                    }
                    fill_phase[stage] = phase;
                    filled[stage] = true;
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
                    if (filled[s]) mbar_wait_bounded(&full[s], fill_phase[s], kWaitLimitNs);
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            constexpr uint32_t IDESC = idesc_bf16_f32(BM, BN);
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
                for (int kq = 0; kq < nk; ++kq) {
                    if (!mbar_wait_bounded(&full[stage], phase, kWaitLimitNs)) {
                        atomicExch(p.err, 3);
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sb = sbase + stage * STAGE_BYTES;
                    const uint64_t a0h = smem_desc_kmajor(sb + OFF_P0, 128, 256);
                    const uint64_t a0l = smem_desc_kmajor(sb + HALF + OFF_P0, 128, 256);
                    const uint64_t b1h = smem_desc_kmajor(sb + OFF_P1, 128, 256);
                    const uint64_t b1l = smem_desc_kmajor(sb + HALF + OFF_P1, 128, 256);
                    const uint32_t accum = kq > 0 ? 1u : 0u;
                    mma_bf16(tmem, a0h, b1h, IDESC, accum);
                    mma_bf16(tmem, a0h, b1l, IDESC, 1u);
                    mma_bf16(tmem, a0l, b1h, IDESC, 1u);
                    const uint64_t a2h = (MODE == PAIR_OPPOSITE_SPIN) ? a0h : smem_desc_kmajor(sb + OFF_P2, 128, 256);
                    const uint64_t a2l = (MODE == PAIR_OPPOSITE_SPIN) ? a0l : smem_desc_kmajor(sb + HALF + OFF_P2, 128, 256);
                    const uint64_t b3h = smem_desc_kmajor(sb + OFF_P3, 128, 256);
                    const uint64_t b3l = smem_desc_kmajor(sb + HALF + OFF_P3, 128, 256);
                    mma_bf16(tmem + BN, a2h, b3h, IDESC, accum);
                    mma_bf16(tmem + BN, a2h, b3l, IDESC, 1u);
                    mma_bf16(tmem + BN, a2l, b3h, IDESC, 1u);
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
            if (*abort_flag) break;
            const int2 ij = p.pairs[u / p.nblocks];
            const int2 xy = p.blocks[u % p.nblocks];
            const int a = xy.x * BM + row;
            const int bbase = xy.y * 128;
            // stage the column energies of this unit while the MMAs run
            for (int c = etid; c < 2 * BN; c += 128) {
                const int b = bbase + c;
                const int lim = (MODE == PAIR_OPPOSITE_SPIN) ? p.vy : p.vx;
                const double* ev = (MODE == PAIR_OPPOSITE_SPIN) ? p.evy : p.evx;
                eb_s[c] = (b < lim && (MODE == PAIR_OPPOSITE_SPIN || c < BN)) ? ev[b] : 0.0;
            }
            asm volatile("bar.sync 1, 128;\n" ::: "memory");
            if (!mbar_wait_bounded(tmem_full, acc_phase, kWaitLimitNs)) {
                atomicExch(p.err, 4);
                *abort_flag = 1;
                break;
            }
            acc_phase ^= 1;
            tc_fence_after();

            const bool arow = a < p.vx;
            double s_lo = 0.0, s_hi = 0.0, o_lo = 0.0, o_hi = 0.0;   // per column half
            const double eij = (MODE == PAIR_OPPOSITE_SPIN) ? p.eox[ij.x] + p.eoy[ij.y]
                                                            : p.eox[ij.x] + p.eox[ij.y];
            const double ta = arow ? eij - p.evx[a] : 0.0;
            const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                uint32_t r1[32], r2[32];
                tmem_ld32(lane_base + c0, r1);
                tmem_ld32(lane_base + BN + c0, r2);
                tmem_ld_wait();
                if (!arow) continue;
                const bool hi_half = c0 >= 128;
#pragma unroll
                for (int k = 0; k < 32; ++k) {
                    const int c = c0 + k;
                    const float V = __uint_as_float(r1[k]);
                    const float W = __uint_as_float(r2[k]);
                    if (MODE == PAIR_OPPOSITE_SPIN) {
                        if (bbase + c < p.vy) {
                            const double D = ta - eb_s[c];
                            if (fabs(D) >= kDenomSkip) {
                                const double t = (double)(V * V) * recip_nr(D);
                                if (hi_half) s_hi += t; else s_lo += t;
                            }
                        }
                        if (bbase + BN + c < p.vy) {
                            const double D = ta - eb_s[BN + c];
                            if (fabs(D) >= kDenomSkip) {
                                const double t = (double)(W * W) * recip_nr(D);
                                if (hi_half) o_hi += t; else o_lo += t;
                            }
                        }
                    } else {
                        if (bbase + c < p.vx) {
                            const double D = ta - eb_s[c];
                            if (fabs(D) >= kDenomSkip) {
                                const double rD = recip_nr(D);
                                if (MODE == PAIR_RESTRICTED) {
                                    const float vw = fmaf(V, V, fmaf(W, W, -V * W));
                                    const float os = fmaf(V, V, W * W);
                                    if (hi_half) { s_hi += (double)vw * rD; o_hi += (double)os * rD; }
                                    else         { s_lo += (double)vw * rD; o_lo += (double)os * rD; }
                                } else {
                                    const float g = V - W;
                                    const double t = (double)(g * g) * rD;
                                    if (hi_half) s_hi += t; else s_lo += t;
                                }
                            }
                        }
                    }
                }
            }
            // accumulators consumed: hand TMEM back to the MMA warp
            tc_fence_before();
            if (lane == 0) mbar_arrive(tmem_empty);

            // weights: column block z = y (first 128) / y+1 (second 128) vs row block x
            double tot1, tot2;
            if (MODE == PAIR_OPPOSITE_SPIN) {
                tot1 = (s_lo + s_hi) + (o_lo + o_hi);
                tot2 = 0.0;
            } else {
                const int x = xy.x, z0 = xy.y, z1 = xy.y + 1;
                double w0, w1;
                if (MODE == PAIR_RESTRICTED) {
                    const double wp = ij.x < ij.y ? 2.0 : 1.0;
                    w0 = wp * (z0 == x ? 1.0 : 2.0);
                    w1 = wp * (z1 == x ? 1.0 : 2.0);
                } else {
                    w0 = (z0 == x ? 0.5 : 1.0);
                    w1 = (z1 == x ? 0.5 : 1.0);
                }
                tot1 = w0 * s_lo + w1 * s_hi;
                tot2 = 0.5 * (w0 * o_lo + w1 * o_hi);
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
