// Element-wise amplitude pass of the MP2 backward.
//
// Input: a staging block of integrals S[(i - i0, a)][(j, b)] = (ia|jb) for
// the occupied rows i of one block and every j (FP32 from vtile_tc.cuh, or
// FP64 from the FP64 GEMM), 32 x 32 tiles with D = e_i + e_j - e_a - e_b
// (|D| < 1e-12 skipped, reference src/mp2/cholesky_rmp2.cc:139):
//
//   RESTRICTED     V = (ia|jb), W = (ib|ja); t = V/D, amplitude tt = (2V - W)/D,
//                  energy V tt, r = t tt          (dE/dB = 4 Gamma)
//   SAME_SPIN      g = V - W, amplitude t = g/D, energy g t / 4, r = t^2 / 4
//                                                  (dE/dB = 2 Gamma)
//   OPPOSITE_SPIN  X alpha, Y beta; amplitude t = V/D, energy V t, r = t^2
//                  (dE/dB_alpha = 2 Gamma_alpha, dE/dB_beta = 2 Gamma_beta)
//
// The energies are those of reference src/mp2/cholesky_rmp2.cc:135-151 and
// src/mp2/cholesky_ump2.cc:316-346, :436-453 summed over ordered pairs.
// Gamma = amplitude x B is formed afterwards by a GEMM with K = (j, b); this
// pass writes the amplitude operand of that GEMM: BF16 hi/lo in the blocked
// K-major layout of the tensor-core Gamma kernel (SPLIT), or FP64 row-major
// [(i - i0, a)][(j, b)] for the FP64 GEMM.  With SPLIT it can also write the
// transposed operand [(j, b)][(i - i0, a)]: Gamma_beta of the opposite-spin
// pass, or, for the symmetric modes (t^{ji}_{ba} = t^{ij}_{ab}), the rows j of
// a block pair (I, J) whose mirror (J, I) is not computed.
// One CTA of 256 threads takes one pair (i, j) and walks its 32 x 32 tiles of
// (a, b), row block outer, loading the next tile while it works on the
// current one; the pair's energy, its row sums
// sum_b r (per a), column sums sum_a r (per b) and total sum r go to per-pair
// buffers, each written by one thread, and deps_*_kernel turn them into
// dE/de (+r on a and b, -r on i and j) in a fixed order.
#pragma once

#include <cuda_bf16.h>

#include <type_traits>

#include "cd_common.cuh"
#include "sm100_ptx.cuh"

namespace mshqc_cd {

enum AmpMode { AMP_RESTRICTED = 0, AMP_SAME_SPIN = 1, AMP_OPPOSITE_SPIN = 2 };

struct AmpElemArgs {
    const void* S;          // float (SPLIT) or double
    long long ldS;          // row length of S
    int rsx;                // rows per occupied i in S and in the output (multiple of 32)
    int csy;                // columns per occupied j in S
    int ksy;                // output K per occupied j (multiple of 32, <= csy)
    int ox, oy, vx, vy, i0, nbi;   // oy: all column orbitals (pair index i * oy + j)
    int j0, nbj;            // the column orbitals of this block: j0 .. j0 + nbj - 1
    double wgt;             // weight of the pair sums (2 when the mirror block (J, I) is skipped)
    const double* eox; const double* evx;   // energies of the row spin
    const double* eoy; const double* evy;   // of the column spin
    uint16_t* Ahi; uint16_t* Alo; long long nkA;  // SPLIT: rows R = ii*rsx + a, K = jj*ksy + b (nkA = K / 16)
    uint16_t* Thi; uint16_t* Tlo; long long nkT;  // SPLIT, optional transpose: rows jj*ksy + b, K = ii*rsx + a
    double* A64; long long ldA;                   // FP64: [R][K], K = jj*ksy + b
    double* partial;        // [ox * oy] energy of each pair (i, j), i over all row orbitals
    double* prow;           // [ox * oy][rsx] sum_b r per pair and row a (or null)
    double* pcol;           // [ox * oy][ksy] sum_a r per pair and column b (or null)
    double* pocc;           // [ox * oy] sum_ab r per pair (or null)
    // nchunk > 1: each pair's row tiles are split over nchunk CTAs (CTA
    // lp * nchunk + c takes chunk c of local pair lp = ii * nbj + jj); their
    // column sums, energies and totals go to cpcol [lp][c][ksy], cpart and
    // cpocc [lp][c], and amp_chunks_combine_kernel adds the chunks in order
    int nchunk;
    double* cpcol; double* cpart; double* cpocc;
    // tri: a diagonal block pair of the symmetric modes with only its pairs
    // ii <= jj (nbi == nbj, local pairs in the order of vtile_pair): an
    // off-diagonal pair stands for (i, j) and (j, i) -- weight 2 -- and its
    // transposed amplitudes go into the same operand (Thi / Tlo = Ahi / Alo)
    int tri;
};

namespace amp_detail {
// local pair lp -> (ii, jj), row-major or the upper triangle (see tri)
__device__ __forceinline__ void local_pair(const AmpElemArgs& p, int lp, int& ii, int& jj) {
    if (!p.tri) {
        ii = lp / p.nbj;
        jj = lp % p.nbj;
        return;
    }
    int r = lp, i = 0;
    while (r >= p.nbi - i) {
        r -= p.nbi - i;
        ++i;
    }
    ii = i;
    jj = i + r;
}
}  // namespace amp_detail

namespace amp_detail {
// blocked K-major element offset of (row R, column k) in the operand layout
// of the Gamma kernel: 128-row blocks, each holding its nkc 16-wide K chunks
// one after the other (so consecutive K chunks of a tile are one copy), 8 x 8
// core matrices inside a 128 x 16 chunk
__device__ __forceinline__ long long blocked_offset(long long R, long long k, long long nkc) {
    return ((R >> 7) * nkc + (k >> 4)) * 2048 + (((R & 127) >> 3) * 16 + ((k & 15) >> 3) * 8 + (R & 7)) * 8 +
           (k & 7);
}

// eight consecutive-k values -> one 16-byte hi row and one 16-byte lo row
__device__ __forceinline__ void store_hilo8(const double* t, uint16_t* hi, uint16_t* lo) {
    uint32_t wh[4], wl[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const __nv_bfloat16 h0 = __double2bfloat16(t[2 * e]), h1 = __double2bfloat16(t[2 * e + 1]);
        const __nv_bfloat16 l0 = __double2bfloat16(t[2 * e] - (double)__bfloat162float(h0));
        const __nv_bfloat16 l1 = __double2bfloat16(t[2 * e + 1] - (double)__bfloat162float(h1));
        wh[e] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        wl[e] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
    }
    *reinterpret_cast<uint4*>(hi) = make_uint4(wh[0], wh[1], wh[2], wh[3]);
    *reinterpret_cast<uint4*>(lo) = make_uint4(wl[0], wl[1], wl[2], wl[3]);
}
}  // namespace amp_detail

template <int MODE, bool SPLIT>
__global__ void __launch_bounds__(256, 4) amp_elem_kernel(AmpElemArgs p) {
    using TS = typename std::conditional<SPLIT, float, double>::type;
    constexpr bool kW = MODE != AMP_OPPOSITE_SPIN;   // (ib|ja) needed
    __shared__ TS Vt[32][33];
    __shared__ TS Wt[kW ? 32 : 1][33];
    __shared__ double T[32][33];
    __shared__ double colpart[8][33];
    __shared__ double red_e[8], red_r[8];
    const TS* S = static_cast<const TS*>(p.S);
    const int ta = p.rsx / 32, tb = p.ksy / 32;
    const int R = p.nchunk > 1 ? p.nchunk : 1;
    const int lp = (int)(blockIdx.x / R), ch = (int)(blockIdx.x % R);
    int ii, jj;
    amp_detail::local_pair(p, lp, ii, jj);
    const double wgt = p.tri ? (ii < jj ? 2.0 : 1.0) : p.wgt;
    const bool write_t = p.Thi != nullptr && !(p.tri && ii == jj);
    // FP64 operand of a diagonal block pair: the (j, i) amplitudes go into A64
    // as the transposes of the (i, j) ones
    const bool write_t64 = !SPLIT && p.tri && ii != jj;
    const int xb0 = ch * ta / R, xb1 = (ch + 1) * ta / R;   // this CTA's row tiles
    const int i = p.i0 + ii, j = p.j0 + jj;
    const long long pair = (long long)i * p.oy + j;          // over all occupied rows
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    const double eij = p.eox[i] + p.eoy[j];
    double* prow = p.prow ? p.prow + pair * p.rsx : nullptr;
    double* pcol = !p.pcol ? nullptr
                   : R == 1 ? p.pcol + pair * p.ksy
                            : p.cpcol + ((long long)lp * R + ch) * p.ksy;
    const TS* Srow = S + (long long)ii * p.rsx * p.ldS + (long long)jj * p.csy;
    // this thread's four elements of tile (a0, b0): rows ty + 8k, column tx
    // (V); the transposed tile (b0, a0) for W
    auto load_tile = [&](int a0, int b0, TS (&v)[4], TS (&w)[4]) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int r = ty + 8 * k;
            // streaming loads: the staging is read here and never again
            v[k] = __ldcs(Srow + (long long)(a0 + r) * p.ldS + b0 + tx);
            if (kW) w[k] = __ldcs(Srow + (long long)(b0 + r) * p.ldS + a0 + tx);
        }
    };
    TS vn[4], wn[4];
    if (xb0 < xb1) load_tile(xb0 * 32, 0, vn, wn);
    double esum = 0.0, rtot = 0.0;
    // row blocks outer, column blocks inner: a thread's rows stay fixed over
    // the inner loop, so their sums over b stay in registers; the column sums
    // of a tile are reduced across the warps and added to pcol in xb order
    for (int xb = xb0; xb < xb1; ++xb) {
        const int a0 = xb * 32;
        double rsum[4] = {0.0, 0.0, 0.0, 0.0};
        for (int yb = 0; yb < tb; ++yb) {
            const int b0 = yb * 32;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                Vt[ty + 8 * k][tx] = vn[k];
                if (kW) Wt[ty + 8 * k][tx] = wn[k];
            }
            // the next tile's loads overlap this tile's arithmetic and stores
            if (yb + 1 < tb)
                load_tile(a0, b0 + 32, vn, wn);
            else if (xb + 1 < xb1)
                load_tile(a0 + 32, 0, vn, wn);
            __syncthreads();
            double cp = 0.0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int r = ty * 4 + k;
                const int a = a0 + r, b = b0 + tx;
                double amp = 0.0, rr = 0.0;
                if (a < p.vx && b < p.vy) {
                    const double D = eij - p.evx[a] - p.evy[b];
                    if (fabs(D) >= kDenomSkip) {
                        const double V = (double)Vt[r][tx];
                        const double rD = SPLIT ? sm100::recip_nr(D) : 1.0 / D;
                        if (MODE == AMP_RESTRICTED) {
                            const double W = (double)Wt[tx][r];
                            const double t = V * rD;
                            amp = (2.0 * V - W) * rD;
                            rr = t * amp;
                            esum = fma(V, amp, esum);
                        } else if (MODE == AMP_SAME_SPIN) {
                            const double W = (double)Wt[tx][r];
                            const double g = V - W;
                            amp = g * rD;
                            rr = 0.25 * amp * amp;
                            esum = fma(0.25 * g, amp, esum);
                        } else {
                            amp = V * rD;
                            rr = amp * amp;
                            esum = fma(V, amp, esum);
                        }
                    }
                }
                T[r][tx] = amp;
                rsum[k] += rr;
                cp += rr;
                if (!SPLIT) p.A64[((long long)ii * p.rsx + a) * p.ldA + (long long)jj * p.ksy + b] = amp;
            }
            rtot += cp;
            colpart[ty][tx] = cp;
            __syncthreads();
            if (SPLIT) {
                // 32 rows x 4 groups of 8 K = 128 core-matrix rows per operand
                if (threadIdx.x < 128) {
                    const int r = threadIdx.x >> 2, g = threadIdx.x & 3;
                    const long long R = (long long)ii * p.rsx + a0 + r;
                    const long long kc = (long long)jj * p.ksy + b0 + g * 8;
                    const long long off = amp_detail::blocked_offset(R, kc, p.nkA);
                    amp_detail::store_hilo8(&T[r][g * 8], p.Ahi + off, p.Alo + off);
                } else if (write_t) {
                    const int w = threadIdx.x - 128;
                    const int r = w >> 2, g = w & 3;   // r: b offset, g: group of 8 a
                    const long long R = (long long)jj * p.ksy + b0 + r;
                    const long long kc = (long long)ii * p.rsx + a0 + g * 8;
                    const long long off = amp_detail::blocked_offset(R, kc, p.nkT);
                    double col[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) col[e] = T[g * 8 + e][r];
                    amp_detail::store_hilo8(col, p.Thi + off, p.Tlo + off);
                }
            }
            if (write_t64) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int rb = ty + 8 * k;   // b offset: row (j, b) of the operand
                    p.A64[((long long)jj * p.ksy + b0 + rb) * p.ldA + (long long)ii * p.rsx + a0 + tx] = T[tx][rb];
                }
            }
            if (pcol && ty == 0) {
                double c = 0.0;
#pragma unroll
                for (int w = 0; w < 8; ++w) c += colpart[w][tx];
                pcol[b0 + tx] = (xb == xb0 ? 0.0 : pcol[b0 + tx]) + wgt * c;
            }
            __syncthreads();   // Vt, Wt, T, colpart are refilled by the next tile
        }
        if (prow) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                double rs = rsum[k];
#pragma unroll
                for (int off = 16; off; off >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, off);
                if (tx == 0) prow[a0 + ty * 4 + k] = wgt * rs;
            }
        }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        esum += __shfl_xor_sync(0xffffffffu, esum, off);
        rtot += __shfl_xor_sync(0xffffffffu, rtot, off);
    }
    if (tx == 0) {
        red_e[ty] = esum;
        red_r[ty] = rtot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double e = 0.0, r = 0.0;
        for (int w = 0; w < 8; ++w) {
            e += red_e[w];
            r += red_r[w];
        }
        if (R == 1) {
            p.partial[pair] = wgt * e;
            if (p.pocc) p.pocc[pair] = wgt * r;
        } else {
            p.cpart[(long long)lp * R + ch] = wgt * e;
            if (p.pocc) p.cpocc[(long long)lp * R + ch] = wgt * r;
        }
    }
}

// The chunk partials of amp_elem_kernel (nchunk > 1) of the nbi x nbj local
// pairs added in chunk order into the per-pair outputs: one thread per
// (local pair, column b); the b == 0 thread also does energy and total.
static __global__ void amp_chunks_combine_kernel(AmpElemArgs p, int npl) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= (long long)npl * p.ksy) return;
    const int lp = (int)(idx / p.ksy), b = (int)(idx % p.ksy);
    const int R = p.nchunk;
    int ii, jj;
    amp_detail::local_pair(p, lp, ii, jj);
    const long long pair = (long long)(p.i0 + ii) * p.oy + p.j0 + jj;
    if (p.pcol) {
        double sc = 0.0;
        for (int c = 0; c < R; ++c) sc += p.cpcol[((long long)lp * R + c) * p.ksy + b];
        p.pcol[pair * p.ksy + b] = sc;
    }
    if (b == 0) {
        double e = 0.0, r = 0.0;
        for (int c = 0; c < R; ++c) {
            e += p.cpart[(long long)lp * R + c];
            if (p.pocc) r += p.cpocc[(long long)lp * R + c];
        }
        p.partial[pair] = e;
        if (p.pocc) p.pocc[pair] = r;
    }
}

// dE/de from the per-pair sums, in a fixed order (no atomics):
// deps_x[ox + a] += sum_pairs prow, deps_y[oy + b] += sum_pairs pcol,
// deps_x[i] -= sum_j pocc[i][j], deps_y[j] -= sum_i pocc[i][j]
static __global__ void deps_rows_kernel(const double* __restrict__ prow, long long npairs, int rsx, int v,
                                        double* __restrict__ dvir) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= v) return;
    double s = 0.0;
    for (long long q = 0; q < npairs; ++q) s += prow[q * rsx + a];
    dvir[a] += s;
}

// (dx and dy may be the same array: thread t touches only element t of each)
static __global__ void deps_occ_kernel(const double* __restrict__ pocc, int ox, int oy, double* __restrict__ dx,
                                       double* __restrict__ dy) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ox) {
        double s = 0.0;
        for (int j = 0; j < oy; ++j) s += pocc[(long long)t * oy + j];
        dx[t] -= s;
    }
    if (t < oy) {
        double s = 0.0;
        for (int i = 0; i < ox; ++i) s += pocc[(long long)i * oy + t];
        dy[t] -= s;
    }
}

}  // namespace mshqc_cd
