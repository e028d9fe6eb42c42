// Pivoted incomplete Cholesky decomposition of the AO ERI matrix on the GPU,
// FP64 throughout: CholeskyERI::decompose (reference
// src/integrals/cholesky_eri.cc:40-149).
//
// E[(ij)][(kl)] = (ij|kl), composite index ij = i N + j.  Diagonal
// D_ij = (ij|ij); each step takes the first index of the largest D (:155-167),
// stops when it is below the threshold, forms
//   L_new[ij] = (E[ij][p] - sum_k L_k[ij] L_k[p]) / sqrt(D_p)   (:169-203)
// (no division when sqrt(D_p) <= 1e-12), then D -= L_new^2 clamped at 0
// (:108-109).  Products and differences are rounded separately, in the
// reference's order.  The vectors become the context's stored vectors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cd_common.cuh"
#include "cd_internal.h"
#include "../../include/mshqc_ao.h"

namespace mshqc_cd {
namespace {

__global__ void eri_diag_kernel(const double* __restrict__ eri, int64_t n2, double* __restrict__ D) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < n2) D[e] = eri[e * n2 + e];
}

// first index of the maximum of D (one CTA of 1024 threads)
__global__ void __launch_bounds__(1024) argmax_first_kernel(const double* __restrict__ D, int64_t n,
                                                            int64_t* __restrict__ pivot,
                                                            double* __restrict__ value) {
    __shared__ double sv[1024];
    __shared__ int64_t si[1024];
    double best = -INFINITY;
    int64_t bi = n;
    for (int64_t e = threadIdx.x; e < n; e += 1024)
        if (D[e] > best) {
            best = D[e];
            bi = e;
        }
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int h = 512; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            const double v2 = sv[threadIdx.x + h];
            const int64_t i2 = si[threadIdx.x + h];
            if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && i2 < si[threadIdx.x])) {
                sv[threadIdx.x] = v2;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *pivot = si[0];
        *value = sv[0];
    }
}

__global__ void chol_column_kernel(const double* __restrict__ eri, int64_t n2, const double* __restrict__ L,
                                   int m, int64_t p, double Dp, double* __restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n2) return;
    double val = eri[e * n2 + p];
    for (int k = 0; k < m; ++k) val = __dsub_rn(val, __dmul_rn(L[(int64_t)k * n2 + e], L[(int64_t)k * n2 + p]));
    const double nf = sqrt(Dp);
    out[e] = nf > 1e-12 ? val / nf : val;
}

// integral-direct variant: the column (e|p) arrives in out, is reduced in
// place in the order of src/integrals/cholesky_direct.cc:180-186 and divided
// by sqrt(D_p)
__global__ void chol_direct_column_kernel(const double* __restrict__ L, int m, int64_t n2, int64_t p, double Dp,
                                          double* __restrict__ out) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n2) return;
    double val = out[e];
    for (int k = 0; k < m; ++k) val = __dsub_rn(val, __dmul_rn(L[(int64_t)k * n2 + e], L[(int64_t)k * n2 + p]));
    out[e] = val / sqrt(Dp);
}

// D -= L^2 with the direct variant's clamp: only small negatives (> -1e-10)
// become zero (src/integrals/cholesky_direct.cc:130-134)
__global__ void chol_direct_diag_update_kernel(double* __restrict__ D, const double* __restrict__ Lm, int64_t n2) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n2) return;
    double d = __dsub_rn(D[e], __dmul_rn(Lm[e], Lm[e]));
    if (d < 0.0 && d > -1e-10) d = 0.0;
    D[e] = d;
}

__global__ void chol_diag_update_kernel(double* __restrict__ D, const double* __restrict__ Lm, int64_t n2) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n2) return;
    double d = __dsub_rn(D[e], __dmul_rn(Lm[e], Lm[e]));
    if (d < 0.0) d = 0.0;
    D[e] = d;
}

}  // namespace
}  // namespace mshqc_cd

using namespace mshqc_cd;

extern "C" MSHQC_CD_API int mshqc_cd_cholesky_decompose(mshqc_cd_ctx* ctx, const double* eri, int64_t nbf,
                                                        double threshold, double* L_out, int64_t max_vectors,
                                                        int64_t* n_vectors, int* converged, int where) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (!eri || !n_vectors) return set_error(MSHQC_CD_ERR_ARG, "eri and n_vectors must be non-null");
    if (nbf <= 0) return set_error(MSHQC_CD_ERR_ARG, "nbf must be positive");
    if (!(threshold > 0.0)) return set_error(MSHQC_CD_ERR_ARG, "threshold must be positive");
    if (where != MSHQC_CD_HOST && where != MSHQC_CD_DEVICE)
        return set_error(MSHQC_CD_ERR_ARG, "unknown pointer location");
    DeviceGuard g(ctx->device);
    const int64_t n2 = nbf * nbf;
    ctx->invalidate_all();
    ctx->L_set = false;
    ctx->L_gen = false;
    // the ERI matrix on the device (scratch), the diagonal and the pivot
    CD_ALLOC(ctx->scratch, sizeof(double) * (size_t)(n2 * n2 + n2 + 2), false);
    double* dE = ctx->scratch.as<double>();
    double* D = dE + n2 * n2;
    double* pv = D + n2;   // [0] pivot index (as int64), [1] its value
    if (where == MSHQC_CD_HOST) {
        CD_RC(upload(ctx, dE, eri, sizeof(double) * (size_t)(n2 * n2)));
    } else {
        CD_CUDA(cudaMemcpyAsync(dE, eri, sizeof(double) * (size_t)(n2 * n2), cudaMemcpyDeviceToDevice,
                                ctx->stream));
    }
    CD_RC(check_finite_device(ctx, dE, n2 * n2, "eri"));
    CD_ALLOC(ctx->L, sizeof(double) * (size_t)(n2 * n2), false);   // at most n^2 vectors
    double* L = ctx->L.as<double>();
    const unsigned blocks = (unsigned)cdiv(n2, 256);
    eri_diag_kernel<<<blocks, 256, 0, ctx->stream>>>(dE, n2, D);
    CD_CUDA(cudaGetLastError());
    int64_t m = 0;
    for (; m < n2; ++m) {
        argmax_first_kernel<<<1, 1024, 0, ctx->stream>>>(D, n2, reinterpret_cast<int64_t*>(pv), pv + 1);
        CD_CUDA(cudaGetLastError());
        struct {
            int64_t p;
            double v;
        } h;
        CD_CUDA(cudaMemcpyAsync(&h, pv, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        CD_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h.v < threshold) break;
        chol_column_kernel<<<blocks, 256, 0, ctx->stream>>>(dE, n2, L, (int)m, h.p, h.v, L + m * n2);
        chol_diag_update_kernel<<<blocks, 256, 0, ctx->stream>>>(D, L + m * n2, n2);
        CD_CUDA(cudaGetLastError());
        ctx->launches += 3;
    }
    *n_vectors = m;
    if (converged) *converged = m < n2 ? 1 : 0;
    if (L_out) {
        if (m > max_vectors)
            return set_error(MSHQC_CD_ERR_ARG, "L_out holds " + std::to_string(max_vectors) + " vectors, " +
                                                   std::to_string(m) + " were produced");
        CD_RC(download(ctx, L_out, L, sizeof(double) * (size_t)(m * n2), where));
    }
    ctx->N = nbf;
    ctx->M = m;
    ctx->Mp = round_up(std::max<int64_t>(m, 1), 16);
    ctx->L_set = m > 0;
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}

// Integral-direct pivoted Cholesky (reference src/integrals/cholesky_direct.cc:
// 32-187, DirectCholesky::compute): the ERI diagonal and, per vector, the one
// ERI column of the pivot come from the host AO engine (mshqc_ao_*), the
// pivot search, the column reduction and the diagonal update run on the
// device.  Stops when the largest diagonal is below the threshold or
// negative, or after N^2 / 2 vectors, as the reference does.
extern "C" MSHQC_CD_API int mshqc_cd_cholesky_direct(mshqc_cd_ctx* ctx, const mshqc_ao_basis* basis,
                                                     double threshold, double* L_out, int64_t max_vectors,
                                                     int64_t* n_vectors, int* converged, int where) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (!basis || !n_vectors) return set_error(MSHQC_CD_ERR_ARG, "basis and n_vectors must be non-null");
    if (!(threshold > 0.0)) return set_error(MSHQC_CD_ERR_ARG, "threshold must be positive");
    if (where != MSHQC_CD_HOST && where != MSHQC_CD_DEVICE)
        return set_error(MSHQC_CD_ERR_ARG, "unknown pointer location");
    int64_t nbf = 0;
    if (mshqc_ao_nbf(basis, &nbf) != MSHQC_AO_OK)
        return set_error(MSHQC_CD_ERR_ARG, std::string("basis: ") + mshqc_ao_last_error());
    DeviceGuard g(ctx->device);
    const int64_t n2 = nbf * nbf, vmax = n2 / 2 + 1;
    ctx->invalidate_all();
    ctx->L_set = false;
    ctx->L_gen = false;
    std::vector<double> hcol((size_t)n2);
    if (mshqc_ao_eri_diagonal(basis, hcol.data()) != MSHQC_AO_OK)
        return set_error(MSHQC_CD_ERR_ARG, std::string("ERI diagonal: ") + mshqc_ao_last_error());
    CD_ALLOC(ctx->scratch, sizeof(double) * (size_t)(n2 + 2), false);
    double* D = ctx->scratch.as<double>();
    double* pv = D + n2;
    CD_RC(upload(ctx, D, hcol.data(), sizeof(double) * (size_t)n2));
    CD_ALLOC(ctx->L, sizeof(double) * (size_t)(vmax * n2), false);
    double* L = ctx->L.as<double>();
    const unsigned blocks = (unsigned)cdiv(n2, 256);
    int64_t m = 0;
    bool conv = false;
    for (; m < vmax; ++m) {
        argmax_first_kernel<<<1, 1024, 0, ctx->stream>>>(D, n2, reinterpret_cast<int64_t*>(pv), pv + 1);
        CD_CUDA(cudaGetLastError());
        struct {
            int64_t p;
            double v;
        } h;
        CD_CUDA(cudaMemcpyAsync(&h, pv, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        CD_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h.v < threshold) {   // also a negative largest diagonal
            conv = h.v >= -1e-10;
            break;
        }
        if (mshqc_ao_eri_column(basis, h.p, hcol.data()) != MSHQC_AO_OK)
            return set_error(MSHQC_CD_ERR_ARG, std::string("ERI column: ") + mshqc_ao_last_error());
        CD_RC(upload(ctx, L + m * n2, hcol.data(), sizeof(double) * (size_t)n2));
        chol_direct_column_kernel<<<blocks, 256, 0, ctx->stream>>>(L, (int)m, n2, h.p, h.v, L + m * n2);
        chol_direct_diag_update_kernel<<<blocks, 256, 0, ctx->stream>>>(D, L + m * n2, n2);
        CD_CUDA(cudaGetLastError());
        ctx->launches += 3;
    }
    *n_vectors = m;
    if (converged) *converged = conv ? 1 : 0;
    if (L_out) {
        if (m > max_vectors)
            return set_error(MSHQC_CD_ERR_ARG, "L_out holds " + std::to_string(max_vectors) + " vectors, " +
                                                   std::to_string(m) + " were produced");
        CD_RC(download(ctx, L_out, L, sizeof(double) * (size_t)(m * n2), where));
    }
    ctx->N = nbf;
    ctx->M = m;
    ctx->Mp = round_up(std::max<int64_t>(m, 1), 16);
    ctx->L_set = m > 0;
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}
