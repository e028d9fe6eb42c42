// Blocks of MP2 amplitudes for the consumers of the reference's stored t2
// (CholeskyRMP2Result::t2, read by CholeskyRMP3, src/mp3/cholesky_rmp3.cc:29,
// :89-90; CholeskyUMP2::compute_t2_amplitudes, src/mp2/cholesky_ump2.cc:
// 471-556, whose t2_aa_/t2_bb_/t2_ab_ CholeskyUMP3 reads).  The MP2 path
// itself never stores o^2 v^2 amplitudes; this entry forms any block of
// pairs on request, in FP64:
//   t_ij^ab = (ia|jb) / (e_i + e_j - e_a - e_b),  0 where |D| < 1e-12,
// the reference's convention in every spin block (no antisymmetrization).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "cd_common.cuh"
#include "cd_internal.h"
#include "gemm_f64.cuh"

namespace mshqc_cd {
namespace {

// out[((ii nj + jj) vx + a) vy + b] /= D, zero where |D| < kDenomSkip
__global__ void t2_divide_kernel(double* __restrict__ out, int ni, int nj, int vx, int vy, int i0, int j0,
                                 const double* __restrict__ eox, const double* __restrict__ evx,
                                 const double* __restrict__ eoy, const double* __restrict__ evy) {
    const int64_t n = (int64_t)ni * nj * vx * vy;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t % vy);
        const int64_t r = t / vy;
        const int a = (int)(r % vx);
        const int64_t p = r / vx;
        const int jj = (int)(p % nj), ii = (int)(p / nj);
        const double D = eox[i0 + ii] + eoy[j0 + jj] - evx[a] - evy[b];
        out[t] = fabs(D) < kDenomSkip ? 0.0 : out[t] / D;
    }
}

}  // namespace
}  // namespace mshqc_cd

using namespace mshqc_cd;

extern "C" MSHQC_CD_API int mshqc_cd_get_t2_block(mshqc_cd_ctx* ctx, int block, int64_t i0, int64_t ni, int64_t j0,
                                                  int64_t nj, double* out, int where) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (!out) return set_error(MSHQC_CD_ERR_ARG, "out is null");
    if (block < 0 || block > 2) return set_error(MSHQC_CD_ERR_ARG, "block must be 0 (alpha-alpha), 1 or 2");
    DeviceGuard g(ctx->device);
    const int sx = block == 1 ? 1 : 0, sy = block == 0 ? 0 : 1;
    for (int s : {sx, sy})
        if (!ctx->spin[s].set)
            return set_error(MSHQC_CD_ERR_STATE, s == 0 ? "alpha orbitals not set" : "beta orbitals not set");
    const int64_t ox = ctx->spin[sx].nocc, oy = ctx->spin[sy].nocc;
    if (i0 < 0 || ni < 1 || i0 + ni > ox || j0 < 0 || nj < 1 || j0 + nj > oy)
        return set_error(MSHQC_CD_ERR_ARG, "pair block outside the occupied orbitals");
    CD_RC(ensure_transform(ctx, sx, MSHQC_CD_FP64));
    if (sy != sx) CD_RC(ensure_transform(ctx, sy, MSHQC_CD_FP64));
    const SpinState& X = ctx->spin[sx];
    const SpinState& Y = ctx->spin[sy];
    const int64_t vx = ctx->N - ox, vy = ctx->N - oy, Mp = ctx->Mp;
    const size_t n = (size_t)(ni * nj * vx * vy);
    double* dst = out;
    if (where != MSHQC_CD_DEVICE) {
        CD_ALLOC(ctx->scratch, n * sizeof(double), false);
        dst = ctx->scratch.as<double>();
    }
    // (ia|jb) for j in the block, one batched GEMM per i: C_jj = B_i B_j^T
    for (int64_t ii = 0; ii < ni; ++ii) {
        GemmF64Args a{};
        a.M = (int)vx;  a.N = (int)vy;  a.K = (int)Mp;  a.batch = (int)nj;
        a.A = X.B64.as<double>() + (i0 + ii) * X.vp * Mp;  a.lda = Mp;  a.sA = 0;
        a.B = Y.B64.as<double>() + j0 * Y.vp * Mp;  a.ldb = Mp;  a.sB = Y.vp * Mp;
        a.C = dst + ii * nj * vx * vy;  a.ldc = vy;  a.sC = vx * vy;
        a.alpha = 1.0;  a.beta = 0.0;
        CD_CUDA(gemm_f64(a, true, true, ctx->stream));
        ctx->launches++;
    }
    const double* ex = X.eps.as<double>();
    const double* ey = Y.eps.as<double>();
    const int blocks = (int)std::min<int64_t>(cdiv((int64_t)n, 256), (int64_t)ctx->num_sms * 8);
    t2_divide_kernel<<<blocks, 256, 0, ctx->stream>>>(dst, (int)ni, (int)nj, (int)vx, (int)vy, (int)i0, (int)j0, ex,
                                                     ex + ox, ey, ey + oy);
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    if (where != MSHQC_CD_DEVICE)
        CD_CUDA(cudaMemcpyAsync(out, dst, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}
