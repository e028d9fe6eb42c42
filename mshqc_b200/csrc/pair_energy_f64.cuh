// Fused FP64 pair-energy kernel (the FP64 path of the MP2 pair loop).
//
// One CTA = one work unit (pair (i,j), virtual row block A, column block B;
// 64 x 64).  It forms two integral tiles with DMMA, K = Q streamed through
// shared memory, and reduces the energy contributions of the unit without
// writing (ia|jb) or the amplitudes anywhere:
//
//   RESTRICTED / SAME_SPIN  T1[a,b] = (ia|jb) = sum_Q X_i[a,Q] X_j[b,Q]
//                           T2[a,b] = (ib|ja) = sum_Q X_j[a,Q] X_i[b,Q]
//   OPPOSITE_SPIN           T1[a,b] = (ia|jb) with X (alpha) i, Y (beta) j,
//                           T2 = the same for the next 64 columns of b.
//
// Energy per element (D = e_i + e_j - e_a - e_b, |D| < 1e-12 skipped):
//   RESTRICTED    w_AB (V^2 + W^2 - V W) / D,  w_AB = 2 (A<B) or 1 (A=B);
//                 pairs i <= j, pair weight 2 (i<j) / 1 (i=j).  Summed over
//                 the units this is sum_{ij,ab} V(2V - V^T)/D of reference
//                 src/mp2/cholesky_rmp2.cc:135-151 (D is symmetric in a,b).
//   SAME_SPIN     w_AB (V - W)^2 / D, w_AB = 1 (A<B) or 1/2 (A=B); pairs
//                 i < j.  Equals 1/4 sum_{ijab} (g_ijab - g_ijba)^2 / D of
//                 src/mp2/cholesky_ump2.cc:316-346.
//   OPPOSITE_SPIN V^2 / D over all pairs and blocks
//                 (src/mp2/cholesky_ump2.cc:436-453).
// The unit's compensated FP64 sum goes to partial[unit]; a separate
// deterministic reduction forms pair and total energies.
#pragma once

#include "cd_common.cuh"

namespace mshqc_cd {

enum PairMode { PAIR_RESTRICTED = 0, PAIR_SAME_SPIN = 1, PAIR_OPPOSITE_SPIN = 2 };

struct PairF64Args {
    const double* X;   // [ox][vpx][Mp]
    const double* Y;   // [oy][vpy][Mp]   (== X for RESTRICTED / SAME_SPIN)
    int vx, vy;        // virtual counts
    int vpx, vpy;      // padded virtual counts (multiples of 64)
    int Mp;            // padded Q extent (multiple of 16; padding is zero)
    const double* eox; const double* evx;   // occupied / virtual energies of X
    const double* eoy; const double* evy;
    const int2* pairs;  // (i, j) per pair
    const int2* blocks; // (row block, column block) per unit of a pair, 64-blocks
    int nblocks;
    double* partial;    // [npairs * nblocks]
    double* partial2;   // RESTRICTED: opposite-spin part per unit
};

namespace pair_f64_detail {
constexpr int BT = 64;          // tile edge
constexpr int BK = 16;          // Q step
constexpr int SK = BK + 4;      // smem row stride (doubles)
constexpr int SLAB = BT * SK;   // doubles per slab per stage
constexpr int STAGES = 2;
constexpr int THREADS = 256;
constexpr size_t SMEM_BYTES = sizeof(double) * SLAB * 4 * STAGES;
}  // namespace pair_f64_detail

template <int MODE>
__global__ void __launch_bounds__(256, 2) pair_energy_f64_kernel(PairF64Args p) {
    using namespace pair_f64_detail;
    extern __shared__ __align__(16) double smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 2, wn = warp & 3;   // 2 x 4 warps: 32 rows x 16 cols each
    const int64_t unit = blockIdx.x;
    const int pidx = (int)(unit / p.nblocks);
    const int bidx = (int)(unit % p.nblocks);
    const int2 ij = p.pairs[pidx];
    const int2 ab = p.blocks[bidx];
    const int i = ij.x, j = ij.y;
    const int a0 = ab.x * BT, b0 = ab.y * BT;
    const int64_t Mp = p.Mp;

    // slab row bases and number of rows that exist in memory
    const double* s0;  const double* s1;  const double* s2;  const double* s3;
    int r0v, r1v, r2v, r3v;
    if (MODE == PAIR_OPPOSITE_SPIN) {
        s0 = p.X + ((int64_t)i * p.vpx + a0) * Mp;  r0v = BT;
        s1 = p.Y + ((int64_t)j * p.vpy + b0) * Mp;  r1v = BT;
        s2 = s0;                                     r2v = 0;   // not loaded
        s3 = p.Y + ((int64_t)j * p.vpy + b0 + BT) * Mp;
        r3v = (b0 + BT < p.vpy) ? BT : 0;
    } else {
        s0 = p.X + ((int64_t)i * p.vpx + a0) * Mp;  r0v = BT;
        s1 = p.X + ((int64_t)j * p.vpx + b0) * Mp;  r1v = BT;
        s2 = p.X + ((int64_t)j * p.vpx + a0) * Mp;  r2v = BT;
        s3 = p.X + ((int64_t)i * p.vpx + b0) * Mp;  r3v = BT;
    }

    auto load_stage = [&](int st, int k0) {
        double* base = smem + (size_t)st * 4 * SLAB;
        const double* srcs[4] = {s0, s1, s2, s3};
        const int valid[4] = {r0v, r1v, r2v, r3v};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (MODE == PAIR_OPPOSITE_SPIN && s == 2) continue;
            double* sm = base + s * SLAB;
#pragma unroll
            for (int c = tid; c < BT * (BK / 2); c += THREADS) {
                const int r = c >> 3, kc = (c & 7) * 2;
                const bool ok = r < valid[s];
                const double* src = ok ? srcs[s] + (int64_t)r * Mp + k0 + kc : srcs[0];
                cp_async16(sm + r * SK + kc, src, ok ? 16 : 0);
            }
        }
    };

    double acc1[4][2][2], acc2[4][2][2];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 2; ++y) acc1[x][y][0] = acc1[x][y][1] = acc2[x][y][0] = acc2[x][y][1] = 0.0;

    const int nk = p.Mp / BK;
    load_stage(0, 0);
    cp_async_commit();
    for (int kt = 0; kt < nk; ++kt) {
        const int st = kt & 1;
        if (kt + 1 < nk) load_stage(st ^ 1, (kt + 1) * BK);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const double* b = smem + (size_t)st * 4 * SLAB;
        const double* P0 = b;
        const double* P1 = b + SLAB;
        const double* P2 = (MODE == PAIR_OPPOSITE_SPIN) ? b : b + 2 * SLAB;
        const double* P3 = b + 3 * SLAB;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            const int kq = kk + (lane & 3);
            double a1[4], a2[4], b1[2], b2[2];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const int r = wm * 32 + x * 8 + (lane >> 2);
                a1[x] = P0[r * SK + kq];
                a2[x] = P2[r * SK + kq];
            }
#pragma unroll
            for (int y = 0; y < 2; ++y) {
                const int r = wn * 16 + y * 8 + (lane >> 2);
                b1[y] = P1[r * SK + kq];
                b2[y] = P3[r * SK + kq];
            }
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 2; ++y) {
                    dmma_8x8x4(acc1[x][y][0], acc1[x][y][1], a1[x], b1[y]);
                    dmma_8x8x4(acc2[x][y][0], acc2[x][y][1], a2[x], b2[y]);
                }
        }
        __syncthreads();
    }

    // ---- epilogue: energy contributions of this unit -------------------
    KSum sum, sum2;
    sum.init();
    sum2.init();
    if (MODE == PAIR_OPPOSITE_SPIN) {
        const double eij = p.eox[i] + p.eoy[j];
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            const int a = a0 + wm * 32 + x * 8 + (lane >> 2);
            if (a >= p.vx) continue;
            const double ea = p.evx[a];
#pragma unroll
            for (int y = 0; y < 2; ++y)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int c = wn * 16 + y * 8 + 2 * (lane & 3) + e;
                    const int bA = b0 + c, bB = b0 + BT + c;
                    if (bA < p.vy) {
                        const double D = eij - ea - p.evy[bA];
                        const double V = acc1[x][y][e];
                        if (fabs(D) >= kDenomSkip) sum.add(V * V / D);
                    }
                    if (bB < p.vy) {
                        const double D = eij - ea - p.evy[bB];
                        const double W = acc2[x][y][e];
                        if (fabs(D) >= kDenomSkip) sum.add(W * W / D);
                    }
                }
        }
    } else {
        const double eij = p.eox[i] + p.eox[j];
        const bool diag = (ab.x == ab.y);
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            const int a = a0 + wm * 32 + x * 8 + (lane >> 2);
            if (a >= p.vx) continue;
            const double ea = p.evx[a];
#pragma unroll
            for (int y = 0; y < 2; ++y)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int bb = b0 + wn * 16 + y * 8 + 2 * (lane & 3) + e;
                    if (bb >= p.vx) continue;
                    const double D = eij - ea - p.evx[bb];
                    if (fabs(D) < kDenomSkip) continue;
                    const double V = acc1[x][y][e], W = acc2[x][y][e];
                    if (MODE == PAIR_RESTRICTED) {
                        const double rD = 1.0 / D;
                        sum.add((V * V + W * W - V * W) * rD);
                        sum2.add((V * V + W * W) * rD);
                    } else
                        sum.add((V - W) * (V - W) / D);
                }
        }
        // block weight applied to the whole unit below
        if (MODE == PAIR_RESTRICTED) {
            const double w = (diag ? 1.0 : 2.0) * (i < j ? 2.0 : 1.0);
            sum.s *= w;
            sum.c *= w;
            // opposite-spin part: sum over (a,b) and (b,a) of V_ab^2 is (V^2 + W^2)
            // once per off-diagonal element, half of it on a diagonal block
            sum2.s *= 0.5 * w;
            sum2.c *= 0.5 * w;
        } else {
            const double w = diag ? 0.5 : 1.0;
            sum.s *= w;
            sum.c *= w;
        }
    }

    warp_reduce_ksum(sum);
    if (MODE == PAIR_RESTRICTED) warp_reduce_ksum(sum2);
    __shared__ double red_s[2][8], red_c[2][8];
    if (lane == 0) {
        red_s[0][warp] = sum.s;
        red_c[0][warp] = sum.c;
        red_s[1][warp] = sum2.s;
        red_c[1][warp] = sum2.c;
    }
    __syncthreads();
    if (tid < (MODE == PAIR_RESTRICTED ? 2 : 1)) {
        KSum t;
        t.init();
        for (int w = 0; w < 8; ++w) {
            t.add(red_s[tid][w]);
            t.c += red_c[tid][w];
        }
        (tid == 0 ? p.partial : p.partial2)[unit] = t.value();
    }
}

// Deterministic compensated reduction of unit partials into per-pair sums
// (one thread per pair, units in order) ...
static __global__ void reduce_pairs_kernel(const double* __restrict__ partial, int npairs, int nblocks,
                                    double* __restrict__ pair_sum) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    KSum s;
    s.init();
    const double* src = partial + (int64_t)p * nblocks;
    for (int b = 0; b < nblocks; ++b) s.add(src[b]);
    pair_sum[p] = s.value();
}

// ... and of per-pair sums into one total (single CTA of 256 threads, fixed
// order: strided per-thread sums, then a fixed tree).
static __global__ void reduce_total_kernel(const double* __restrict__ x, int n, double* __restrict__ out) {
    __shared__ double ss[256], sc[256];
    KSum s;
    s.init();
    for (int k = threadIdx.x; k < n; k += 256) s.add(x[k]);
    ss[threadIdx.x] = s.s;
    sc[threadIdx.x] = s.c;
    __syncthreads();
    if (threadIdx.x == 0) {
        KSum t;
        t.init();
        for (int k = 0; k < 256; ++k) {
            t.add(ss[k]);
            t.c += sc[k];
        }
        *out = t.value();
    }
}

}  // namespace mshqc_cd
