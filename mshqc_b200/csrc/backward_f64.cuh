// FP64 amplitude pass of the MP2 backward (restricted closed shell).
//
// One CTA = one unit (i, j, virtual row block A, column block B; 64 x 64) of
// the ordered pairs i in [i0, i0+bi), all j.  With DMMA it forms
//   T1[a,b] = (ia|jb),  T2[a,b] = (ib|ja)
// and from them, per element (D = e_i + e_j - e_a - e_b, |D| < 1e-12 skipped):
//   t  = T1 / D,   tt = (2 T1 - T2) / D          (dE/d(ia|jb) = 2 tt)
//   tile_out[(i-i0), a, (j, b)] = tt              (staging for Gamma = tt . B)
//   energy += T1 tt ;  r = t tt
//   dE/de_a += r, dE/de_b += r (virtual), dE/de_i -= r, dE/de_j -= r (occupied)
// Summed over all ordered pairs these are E and dE/de of
// E = sum_{ij,ab} (ia|jb)(2(ia|jb) - (ib|ja))/D (reference
// src/mp2/cholesky_rmp2.cc:135-151).
#pragma once

#include "cd_common.cuh"
#include "pair_energy_f64.cuh"

namespace mshqc_cd {

struct AmpF64Args {
    const double* X;        // [o][vp][Mp]
    int o, v, vp, Mp;
    int i0, bi;             // occupied row block
    const double* eo; const double* ev;
    double* amp;            // [bi][vp][o*vp]
    double* deps;           // [N]: occupied first, then virtual (atomic accumulation)
    double* partial;        // per unit energy [bi*o*nb*nb]
    int nb;                 // vp / 64
};

__global__ void __launch_bounds__(256, 2) amp_f64_kernel(AmpF64Args p) {
    using namespace pair_f64_detail;
    extern __shared__ __align__(16) double smem[];
    __shared__ double rsum[BT], csum[BT];
    __shared__ double red[8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 2, wn = warp & 3;
    const int64_t unit = blockIdx.x;
    const int nbb = p.nb * p.nb;
    const int pr = (int)(unit / nbb);            // pair index: (i - i0) * o + j
    const int bb = (int)(unit % nbb);
    const int ii = pr / p.o, j = pr % p.o, i = p.i0 + ii;
    const int ax = bb / p.nb, by = bb % p.nb;
    const int a0 = ax * BT, b0 = by * BT;
    const int64_t Mp = p.Mp;
    const double* s0 = p.X + ((int64_t)i * p.vp + a0) * Mp;
    const double* s1 = p.X + ((int64_t)j * p.vp + b0) * Mp;
    const double* s2 = p.X + ((int64_t)j * p.vp + a0) * Mp;
    const double* s3 = p.X + ((int64_t)i * p.vp + b0) * Mp;

    if (tid < BT) {
        rsum[tid] = 0.0;
        csum[tid] = 0.0;
    }

    auto load_stage = [&](int st, int k0) {
        double* base = smem + (size_t)st * 4 * SLAB;
        const double* srcs[4] = {s0, s1, s2, s3};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            double* sm = base + s * SLAB;
#pragma unroll
            for (int c = tid; c < BT * (BK / 2); c += THREADS) {
                const int r = c >> 3, kc = (c & 7) * 2;
                cp_async16(sm + r * SK + kc, srcs[s] + (int64_t)r * Mp + k0 + kc, 16);
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
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            const int kq = kk + (lane & 3);
            double a1[4], a2[4], b1[2], b2[2];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const int r = wm * 32 + x * 8 + (lane >> 2);
                a1[x] = b[r * SK + kq];
                a2[x] = b[2 * SLAB + r * SK + kq];
            }
#pragma unroll
            for (int y = 0; y < 2; ++y) {
                const int r = wn * 16 + y * 8 + (lane >> 2);
                b1[y] = b[SLAB + r * SK + kq];
                b2[y] = b[3 * SLAB + r * SK + kq];
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

    const double eij = p.eo[i] + p.eo[j];
    const int64_t ldo = (int64_t)p.o * p.vp;
    double* out = p.amp + ((int64_t)ii * p.vp) * ldo + (int64_t)j * p.vp;
    double esum = 0.0, rtot = 0.0;
#pragma unroll
    for (int x = 0; x < 4; ++x) {
        const int r = wm * 32 + x * 8 + (lane >> 2);
        const int a = a0 + r;
        const double ea = a < p.v ? p.ev[a] : 0.0;
        double rrow = 0.0;
#pragma unroll
        for (int y = 0; y < 2; ++y)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int c = wn * 16 + y * 8 + 2 * (lane & 3) + e;
                const int bcol = b0 + c;
                double tt = 0.0;
                if (a < p.v && bcol < p.v) {
                    const double D = eij - ea - p.ev[bcol];
                    if (fabs(D) >= kDenomSkip) {
                        const double V = acc1[x][y][e], W = acc2[x][y][e];
                        const double rD = 1.0 / D;
                        tt = (2.0 * V - W) * rD;
                        const double rr = V * rD * tt;
                        esum = fma(V, tt, esum);
                        rrow += rr;
                        atomicAdd(&csum[c], rr);
                    }
                }
                out[(int64_t)a * ldo + bcol] = tt;
            }
        // row sums: lanes sharing lane>>2 hold the same row
        rrow += __shfl_xor_sync(0xffffffffu, rrow, 1);
        rrow += __shfl_xor_sync(0xffffffffu, rrow, 2);
        if ((lane & 3) == 0) atomicAdd(&rsum[r], rrow);
        rtot += ((lane & 3) == 0) ? rrow : 0.0;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        esum += __shfl_xor_sync(0xffffffffu, esum, off);
        rtot += __shfl_xor_sync(0xffffffffu, rtot, off);
    }
    __shared__ double rt[8];
    if (lane == 0) {
        red[warp] = esum;
        rt[warp] = rtot;
    }
    __syncthreads();
    if (tid < BT) {
        if (a0 + tid < p.v) atomicAdd(&p.deps[p.o + a0 + tid], rsum[tid]);
        if (b0 + tid < p.v) atomicAdd(&p.deps[p.o + b0 + tid], csum[tid]);
    }
    if (tid == 0) {
        double e = 0.0, rr = 0.0;
        for (int w = 0; w < 8; ++w) {
            e += red[w];
            rr += rt[w];
        }
        p.partial[unit] = e;
        atomicAdd(&p.deps[i], -rr);
        atomicAdd(&p.deps[j], -rr);
    }
}

}  // namespace mshqc_cd
