// FP64 MO vectors -> BF16 hi/lo pair in the core-matrix blocked layout read
// by the tensor-core pair kernel (pair_energy_tc.cuh):
//   hi = bf16(x), lo = bf16(x - hi); x = hi + lo + O(2^-17 |x|).
// Out-of-range rows (a >= v) and columns (Q >= M) are written as zeros, so
// the whole allocation is defined after one pass.
#pragma once

#include <cuda_bf16.h>

#include "cd_common.cuh"

namespace mshqc_cd {

// src: [o][vp][Mp] FP64 (padded, zeros outside v x M)
// dst: [o][nqc][rows][16] BF16 bits, blocked as (a/8, (Q%16)/8, a%8, Q%8)
static __global__ void split_bf16_blocked_kernel(const double* __restrict__ src, int64_t vp, int64_t Mp,
                                                 int v, int M, int64_t o, int64_t nqc, int64_t rows,
                                                 uint16_t* __restrict__ hi, uint16_t* __restrict__ lo) {
    // one thread = one core-matrix row: 8 consecutive Q of one a
    const int64_t total = o * nqc * rows * 2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        // t enumerates (i, qc, g, kk, r) with r fastest
        const int64_t r = t & 7;
        const int64_t kk = (t >> 3) & 1;
        const int64_t rest = t >> 4;               // (i, qc, g)
        const int64_t ngrp = rows / 8;
        const int64_t g = rest % ngrp;
        const int64_t iq = rest / ngrp;             // i * nqc + qc
        const int64_t qc = iq % nqc, i = iq / nqc;
        const int64_t a = g * 8 + r;
        const int64_t q0 = qc * 16 + kk * 8;
        uint16_t h[8], l[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            double x = 0.0;
            if (a < v && q0 + e < M) x = src[(i * vp + a) * Mp + q0 + e];
            const __nv_bfloat16 bh = __double2bfloat16(x);
            const __nv_bfloat16 bl = __double2bfloat16(x - (double)__bfloat162float(bh));
            h[e] = __bfloat16_as_ushort(bh);
            l[e] = __bfloat16_as_ushort(bl);
        }
        const int64_t off = t * 8;   // == iq*rows*16 + (g*16 + kk*8 + r)*8
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
