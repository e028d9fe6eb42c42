// Integral tiles of the MP2 backward on the tensor cores (tcgen05):
//
//   S[(i - i0, a)][(j, b)] = (ia|jb) = sum_Q B^Q_ia B^Q_jb     (FP32)
//
// for the occupied rows i of one block and all j, every tile computed once.
// Operands are the exact fixed-point hi/lo of split_bf16.cuh in the blocked
// layout of pair_energy_tc.cuh; per 16-wide Q step three 128x256x16 MMAs
// accumulate the hi*hi' and the hi*lo' + lo*hi' integers exactly in two TMEM
// accumulators (columns [0,256) and [256,512)), and the epilogue recovers
//   (ia|jb) = u_ia u_jb (hh + x / 256)
// in FP64, substitutes the exact (ia|ia) for i = j, a = b, and stores it
// rounded to FP32 into the row-major staging matrix S (row length o * VR).
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
    const uint16_t* Xhi; const uint16_t* Xlo;   // blocked fixed-point operands
    const int* ex;                              // row exponents [o][rows]
    const double* diag;                         // exact (ia|ia) [o][rows]
    int rows;               // allocated rows per occupied orbital (operand layout)
    int nqc;                // 16-wide Q chunks
    int o, v, VR, i0, nbi;
    int nbx, nby;           // row blocks (128) per orbital, column ranges (256) per orbital
    int VS;                 // staging columns per orbital j (nby * 256 >= VR)
    float* S;               // staging [nbi * VR][o * VS]
    int* err;
};

namespace vtile_tc {
constexpr int BM = 128, BN = 256, KC = 16, STAGES = 8, THREADS = 192;
constexpr uint32_t SLAB_A = BM * KC * 2;     // 4 KB
constexpr uint32_t SLAB_B = BN * KC * 2;     // 8 KB
constexpr uint32_t OFF_AH = 0, OFF_AL = SLAB_A, OFF_BH = 2 * SLAB_A, OFF_BL = 2 * SLAB_A + SLAB_B;
constexpr uint32_t STAGE_BYTES = 2 * (SLAB_A + SLAB_B);   // 24 KB
constexpr uint32_t SMEM_DATA = STAGES * STAGE_BYTES;      // 192 KB
constexpr size_t SMEM_BYTES = SMEM_DATA + 1024 + 256 + BN * 8;
constexpr uint64_t kWaitLimitNs = 2000000000ull;
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
    const long long units = (long long)p.nbi * p.o * per_pair;
    const long long first = blockIdx.x, step = gridDim.x;
    const int nk = p.nqc;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t stage = 0, phase = 0, fill_phase = 0, filled = 0;
            for (long long u = first; u < units && !*abort_flag; u += step) {
                const long long pr = u / per_pair, bb = u % per_pair;
                const int i = p.i0 + (int)(pr / p.o), j = (int)(pr % p.o);
                const int x = (int)(bb / p.nby), y = (int)(bb % p.nby);
                const size_t rows = p.rows;
                const uint16_t* ah = p.Xhi + (size_t)i * p.nqc * rows * 16 + (size_t)x * BM * 16;
                const uint16_t* al = p.Xlo + (size_t)i * p.nqc * rows * 16 + (size_t)x * BM * 16;
                const uint16_t* bh = p.Xhi + (size_t)j * p.nqc * rows * 16 + (size_t)y * BN * 16;
                const uint16_t* bl = p.Xlo + (size_t)j * p.nqc * rows * 16 + (size_t)y * BN * 16;
                for (int kq = 0; kq < nk; ++kq) {
                    if (!mbar_wait_bounded(&empty[stage], phase ^ 1, kWaitLimitNs)) {
                        atomicExch(p.err, 21);
                        *abort_flag = 1;
                        break;
                    }
                    uint8_t* sb = smem + stage * STAGE_BYTES;
                    mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                    const size_t k = (size_t)kq * rows * 16;
                    bulk_g2s(sb + OFF_AH, ah + k, SLAB_A, &full[stage]);
                    bulk_g2s(sb + OFF_AL, al + k, SLAB_A, &full[stage]);
                    bulk_g2s(sb + OFF_BH, bh + k, SLAB_B, &full[stage]);
                    bulk_g2s(sb + OFF_BL, bl + k, SLAB_B, &full[stage]);
                    fill_phase = (fill_phase & ~(1u << stage)) | (phase << stage);
                    filled |= 1u << stage;
                    if (++stage == STAGES) { stage = 0; phase ^= 1; }
                }
            }
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
                for (int kq = 0; kq < nk; ++kq) {
                    if (!mbar_wait_bounded(&full[stage], phase, kWaitLimitNs)) {
                        atomicExch(p.err, 23);
                        *abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sb = sbase + stage * STAGE_BYTES;
                    const uint64_t ah = smem_desc_kmajor(sb + OFF_AH, 128, 256);
                    const uint64_t al = smem_desc_kmajor(sb + OFF_AL, 128, 256);
                    const uint64_t bh = smem_desc_kmajor(sb + OFF_BH, 128, 256);
                    const uint64_t bl = smem_desc_kmajor(sb + OFF_BL, 128, 256);
                    const uint32_t acc = kq > 0 ? 1u : 0u;
                    mma_f16(tmem, ah, bh, IDESC, acc);
                    mma_f16(tmem + BN, ah, bl, IDESC, acc);
                    mma_f16(tmem + BN, al, bh, IDESC, 1u);
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
        const long long ldS = (long long)p.o * p.VS;
        uint32_t acc_phase = 0;
        for (long long u = first; u < units; u += step) {
            const long long pr = u / per_pair, bb = u % per_pair;
            const int ii = (int)(pr / p.o), j = (int)(pr % p.o), i = p.i0 + ii;
            const int x = (int)(bb / p.nby), y = (int)(bb % p.nby);
            const int a = x * BM + row, b0 = y * BN;
            for (int c = etid; c < BN; c += 128) {
                const int b = b0 + c;
                cs_s[c] = (b < p.v) ? pow2d(p.ex[(size_t)j * p.rows + b] - kFixedHiBits) : 0.0;
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
            const bool arow = a < p.v;
            const double rs = arow ? pow2d(p.ex[(size_t)i * p.rows + a] - kFixedHiBits) : 0.0;
            const int dcol = (arow && i == j && a >= b0 && a < b0 + BN) ? a - b0 : -1;
            const double dg = dcol >= 0 ? p.diag[(size_t)i * p.rows + a] : 0.0;
            float* dst = p.S + ((long long)ii * p.VR + a) * ldS + (long long)j * p.VS + b0;
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
                    float4* d4 = reinterpret_cast<float4*>(dst + c0);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        d4[k] = make_float4(out[4 * k], out[4 * k + 1], out[4 * k + 2], out[4 * k + 3]);
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

// Element-wise amplitude pass on the staging matrix S (one 32 x 32 tile of
// (a, b) for one pair (i, j) per CTA of 256 threads):
//   V = S[(i,a)][(j,b)],  W = S[(i,b)][(j,a)] = (ib|ja),  D = e_i + e_j - e_a - e_b
//   tt = (2V - W)/D, t = V/D, r = t tt
// writes tt as BF16 hi/lo into the blocked Gamma operand (rows (i-i0, a),
// K = (j, b)), adds +r to dE/de_a, dE/de_b and -r to dE/de_i, dE/de_j, and
// stores the tile's sum of V tt (energy) in partial[tile].
struct AmpElemArgs {
    const float* S;         // [nbi * VR][o * VS]
    int o, v, VR, VS, i0, nbi;
    const double* eo; const double* ev;
    uint16_t* Ahi; uint16_t* Alo;   // blocked, RA = nbi_alloc * VR rows
    long long RA;
    double* deps;           // occupied then virtual
    double* partial;        // [nbi * o * (VR/32)^2]
};

static __global__ void __launch_bounds__(256) amp_elem_kernel(AmpElemArgs p) {
    __shared__ float Vt[32][33], Wt[32][33];
    __shared__ double rs[32], cs[32], red[8], rt[8];
    const int nt = p.VR / 32;
    const long long tile = blockIdx.x;
    const long long pr = tile / ((long long)nt * nt);
    const int tb = (int)(tile % ((long long)nt * nt));
    const int ii = (int)(pr / p.o), j = (int)(pr % p.o), i = p.i0 + ii;
    const int a0 = (tb / nt) * 32, b0 = (tb % nt) * 32;
    const long long ldS = (long long)p.o * p.VS;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    if (threadIdx.x < 32) {
        rs[threadIdx.x] = 0.0;
        cs[threadIdx.x] = 0.0;
    }
    // V tile rows a0.., cols b0..; W tile = S rows (i, b0..), cols (j, a0..)
#pragma unroll
    for (int r = ty; r < 32; r += 8) {
        Vt[r][tx] = p.S[((long long)ii * p.VR + a0 + r) * ldS + (long long)j * p.VS + b0 + tx];
        Wt[r][tx] = p.S[((long long)ii * p.VR + b0 + r) * ldS + (long long)j * p.VS + a0 + tx];
    }
    __syncthreads();
    const double eij = p.eo[i] + p.eo[j];
    // each thread: one row a (= ty*4 + k) ... use 4 rows per thread, column tx
    double esum = 0.0, rtot = 0.0;
    double tt_reg[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = ty * 4 + k;
        const int a = a0 + r, b = b0 + tx;
        double tt = 0.0, rr = 0.0;
        if (a < p.v && b < p.v) {
            const double D = eij - p.ev[a] - p.ev[b];
            if (fabs(D) >= kDenomSkip) {
                const double V = Vt[r][tx], W = Wt[tx][r];
                const double rD = 1.0 / D;
                tt = (2.0 * V - W) * rD;
                rr = V * rD * tt;
                esum = fma(V, tt, esum);
            }
        }
        tt_reg[k] = tt;
        rtot += rr;
        // row sum over the 32 columns (lanes)
        double rsum = rr;
#pragma unroll
        for (int off = 16; off; off >>= 1) rsum += __shfl_xor_sync(0xffffffffu, rsum, off);
        if (tx == 0) rs[r] = rsum;
        atomicAdd(&cs[tx], rr);
    }
    // tt through shared memory, then 16-byte core-matrix rows of the blocked layout
    __syncthreads();
    __shared__ double T[32][33];
#pragma unroll
    for (int k = 0; k < 4; ++k) T[ty * 4 + k][tx] = tt_reg[k];
    __syncthreads();
    // 32 rows x 4 groups of 8 columns = 128 core rows; threads 0..127 write one each
    if (threadIdx.x < 128) {
        const int r = threadIdx.x >> 2, g = threadIdx.x & 3;
        const long long R = (long long)ii * p.VR + a0 + r;
        const long long kcol = (long long)j * p.VR + b0 + g * 8;
        const long long off = (kcol >> 4) * p.RA * 16 + ((R >> 3) * 16 + ((kcol & 15) >> 3) * 8 + (R & 7)) * 8;
        uint32_t wh[4], wl[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const double t0 = T[r][g * 8 + 2 * e], t1 = T[r][g * 8 + 2 * e + 1];
            const __nv_bfloat16 h0 = __double2bfloat16(t0), h1 = __double2bfloat16(t1);
            const __nv_bfloat16 l0 = __double2bfloat16(t0 - (double)__bfloat162float(h0));
            const __nv_bfloat16 l1 = __double2bfloat16(t1 - (double)__bfloat162float(h1));
            wh[e] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
            wl[e] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
        }
        *reinterpret_cast<uint4*>(p.Ahi + off) = make_uint4(wh[0], wh[1], wh[2], wh[3]);
        *reinterpret_cast<uint4*>(p.Alo + off) = make_uint4(wl[0], wl[1], wl[2], wl[3]);
    }
    // reductions
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        esum += __shfl_xor_sync(0xffffffffu, esum, off);
        rtot += __shfl_xor_sync(0xffffffffu, rtot, off);
    }
    if (tx == 0) {
        red[ty] = esum;
        rt[ty] = rtot;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int a = a0 + threadIdx.x, b = b0 + threadIdx.x;
        if (a < p.v && rs[threadIdx.x] != 0.0) atomicAdd(&p.deps[p.o + a], rs[threadIdx.x]);
        if (b < p.v && cs[threadIdx.x] != 0.0) atomicAdd(&p.deps[p.o + b], cs[threadIdx.x]);
    }
    if (threadIdx.x == 0) {
        double e = 0.0, r = 0.0;
        for (int w = 0; w < 8; ++w) {
            e += red[w];
            r += rt[w];
        }
        p.partial[tile] = e;
        if (r != 0.0) {
            atomicAdd(&p.deps[i], -r);
            atomicAdd(&p.deps[j], -r);
        }
    }
}

}  // namespace mshqc_cd
