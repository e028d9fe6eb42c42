// FP64 MO vectors -> row-scaled fixed-point pair (hi, lo) carried in FP16, in
// the core-matrix blocked layout read by the tensor-core pair kernel.
//
// Every MO row r = (i, a) gets one power-of-two scale 2^e_r > max_Q |B^Q_r|.
// With u_r = 2^(e_r - 10):
//     hi = rint(x / u_r)                  integer, |hi| <= 1024
//     lo = rint((x - hi u_r) / (u_r/256))  integer, |lo| <= 128
//     x  = u_r (hi + lo/256) + O(u_r/512)    (2^-18 of the row maximum)
// Integers of magnitude <= 2048 are exact in FP16, every product is an
// integer below 2^21, so the FP32 tensor-core accumulators hold exact integers
// as long as every partial sum stays below 2^24.  The Cauchy-Schwarz bounds
// sqrt(sum hi^2 sum hi'^2) (hi*hi' accumulator) and
// sqrt(sum hi^2 sum lo'^2) + sqrt(sum lo^2 sum hi'^2) (cross accumulator),
// checked on the host from the row norms computed here, guarantee that.  The
// accumulated sums are therefore exact whatever rounding the tensor core
// applies, and the only approximation left is the unbiased round-to-nearest
// quantisation above.  The products of a row with itself (the o*v integrals
// (ia|ia)) are the one place where the dropped lo*lo' term is coherent; their
// exact FP64 values are produced here (diag) and substituted by the kernel.
#pragma once

#include <cuda_fp16.h>

#include "cd_common.cuh"

namespace mshqc_cd {

constexpr int kFixedHiBits = 10;   // |hi| <= 2^10
constexpr double kFixedLoScale = 256.0;   // lo step = u / 256, |lo| <= 128

// One warp per row: exponent, exact diagonal and the norms of hi and lo.
// src: [o][vp][Mp] FP64.  rows (a) beyond v get e = 0 and zeros.
// src2 (may be null): second spin's rows for the opposite-spin diagonal
// sum_Q B_alpha[i][a][Q] * B_beta[i][a][Q] (i < o2, a < v2).
static __global__ void row_scale_kernel(const double* __restrict__ src, int64_t vp, int64_t Mp,
                                        int v, int M, int64_t o, int64_t rows,
                                        int* __restrict__ expo, double* __restrict__ diag,
                                        double* __restrict__ norm_hi, double* __restrict__ norm_lo,
                                        const double* __restrict__ src2, int64_t vp2, int o2, int v2,
                                        double* __restrict__ diag_os) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = wid; r < o * rows; r += nw) {
        const int64_t i = r / rows, a = r % rows;
        if (a >= v) {
            if (lane == 0) {
                expo[r] = 0;
                diag[r] = 0.0;
            }
            continue;
        }
        const double* x = src + (i * vp + a) * Mp;
        double mx = 0.0, d = 0.0;
        for (int q = lane; q < M; q += 32) {
            const double t = x[q];
            mx = fmax(mx, fabs(t));
            d = fma(t, t, d);
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
            d += __shfl_xor_sync(0xffffffffu, d, off);
        }
        int e = 0;
        if (mx > 0.0) {
            frexp(mx, &e);              // mx = f 2^e, 0.5 <= f < 1  ->  2^e > mx
        }
        const double inv_u = ldexp(1.0, kFixedHiBits - e), u = ldexp(1.0, e - kFixedHiBits);
        double nh = 0.0, nl = 0.0;
        for (int q = lane; q < M; q += 32) {
            const double t = x[q];
            const double h = rint(t * inv_u);
            const double l = rint((t - h * u) * inv_u * kFixedLoScale);
            nh = fma(h, h, nh);
            nl = fma(l, l, nl);
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            nh += __shfl_xor_sync(0xffffffffu, nh, off);
            nl += __shfl_xor_sync(0xffffffffu, nl, off);
        }
        double dos = 0.0;
        const bool want_os = src2 && i < o2 && a < v2;
        if (want_os) {
            const double* y = src2 + (i * vp2 + a) * Mp;
            for (int q = lane; q < M; q += 32) dos = fma(x[q], y[q], dos);
#pragma unroll
            for (int off = 16; off; off >>= 1) dos += __shfl_xor_sync(0xffffffffu, dos, off);
        }
        if (lane == 0) {
            expo[r] = e;
            diag[r] = d;
            norm_hi[r] = nh;
            norm_lo[r] = nl;
            if (want_os) diag_os[i * rows + a] = dos;
        }
    }
}

// src: [o][vp][Mp] FP64 (zeros outside v x M); expo from row_scale_kernel.
// dst, two layouts of FP16 bits, blocked inside a 16-wide Q chunk as
// (a/8, (Q%16)/8, a%8, Q%8) (the canonical K-major no-swizzle UMMA layout):
//  * pair_layout = false (integral tiles of the backward): hi and lo in
//    separate arrays of 256-row blocks, each holding its nqc chunks one after
//    the other:
//      element (i, a, Q) at ((i*rows/256 + a/256)*nqc + Q/16)*4096
//                           + ((a%256)/8*16 + (Q%16)/8*8 + a%8)*8 + Q%8
//    so a 128-row slab of one chunk is 4 KB and a 256-row slab of consecutive
//    chunks is one contiguous run;
//  * pair_layout = true (fused pair energies): one array of 128-row blocks
//    whose chunks hold the hi slab and then the lo slab of the same rows:
//      hi of (i, a, Q) at ((i*rows/128 + a/128)*nqc + Q/16)*4096
//                         + ((a%128)/8*16 + (Q%16)/8*8 + a%8)*8 + Q%8,
//      lo at the same + 2048,
//    so one contiguous copy brings both halves of a 128-row slab for several
//    chunks, and each chunk's [hi; lo] is a 256-row operand.
// rows is a multiple of 256.
static __global__ void split_fixed_blocked_kernel(const double* __restrict__ src, int64_t vp,
                                                  int64_t Mp, int v, int M, int64_t o, int64_t nqc,
                                                  int64_t rows, const int* __restrict__ expo,
                                                  uint16_t* __restrict__ hi, uint16_t* __restrict__ lo,
                                                  bool pair_layout) {
    // one thread = one core-matrix row: 8 consecutive Q of one a
    const int64_t total = o * nqc * rows * 2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        // t enumerates (i, qc, g, kk, r) with r fastest
        const int64_t r = t & 7;
        const int64_t kk = (t >> 3) & 1;
        const int64_t rest = t >> 4;               // (i*nqc + qc)*ngrp + g
        const int64_t ngrp = rows / 8;
        const int64_t g = rest % ngrp;
        const int64_t iq = rest / ngrp;             // i * nqc + qc
        const int64_t qc = iq % nqc, i = iq / nqc;
        const int64_t a = g * 8 + r;
        const int64_t q0 = qc * 16 + kk * 8;
        const int e = (a < v) ? expo[i * rows + a] : 0;
        const double inv_u = ldexp(1.0, kFixedHiBits - e), u = ldexp(1.0, e - kFixedHiBits);
        uint16_t h[8], l[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            double x = 0.0;
            if (a < v && q0 + k < M) x = src[(i * vp + a) * Mp + q0 + k];
            const double hv = rint(x * inv_u);
            const double lv = rint((x - hv * u) * inv_u * kFixedLoScale);
            h[k] = __half_as_ushort(__double2half(hv));   // exact: |hv| <= 1024
            l[k] = __half_as_ushort(__double2half(lv));   // exact: |lv| <= 128
        }
        const int64_t off = pair_layout
                                ? ((i * (rows / 128) + (g >> 4)) * nqc + qc) * 4096 + ((g & 15) * 16 + kk * 8 + r) * 8
                                : ((i * (rows / 256) + (g >> 5)) * nqc + qc) * 4096 + ((g & 31) * 16 + kk * 8 + r) * 8;
        uint4 vh, vl;
        vh.x = h[0] | (uint32_t(h[1]) << 16); vh.y = h[2] | (uint32_t(h[3]) << 16);
        vh.z = h[4] | (uint32_t(h[5]) << 16); vh.w = h[6] | (uint32_t(h[7]) << 16);
        vl.x = l[0] | (uint32_t(l[1]) << 16); vl.y = l[2] | (uint32_t(l[3]) << 16);
        vl.z = l[4] | (uint32_t(l[5]) << 16); vl.w = l[6] | (uint32_t(l[7]) << 16);
        *reinterpret_cast<uint4*>(hi + off) = vh;
        *reinterpret_cast<uint4*>((pair_layout ? hi + 2048 : lo) + off) = vl;
    }
}

}  // namespace mshqc_cd
