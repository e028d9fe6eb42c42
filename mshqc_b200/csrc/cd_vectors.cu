// Cholesky vectors generated on the device from the synthetic recipe
//
//   L^Q = sigma 10^(-6 Q / M) (X^Q + X^Q^T) / 2,   X^Q_{mu nu} ~ N(0, 1),
//
// for workloads whose FP64 AO vectors do not fit in memory (N = 2000,
// M = 8000 needs 256 GB).  The vectors are never stored: every consumer (the
// forward half transform, the dE/dC_occ transposed transform) asks for
// chunks of Q and they are generated again each time.
//
// For mu < nu one Philox4x32-10 block (the counter-based generator of Salmon,
// Moraes, Dror and Shaw, SC 2011) with key = seed and counter
// (Q N + mu) N + nu gives u1 (first 64 output bits) and u2 (second) and the
// Box-Muller pair r = sqrt(-2 ln u1), X^Q_{mu nu} = r cos(2 pi u2),
// X^Q_{nu mu} = r sin(2 pi u2): two independent N(0, 1) draws, so one
// logarithm and one sincos per symmetric element pair.  X^Q_{mu mu} is the
// cosine member of counter (Q N + mu) N + mu.  mshqc_b200/synthetic.py holds
// the same recipe in numpy (make_vectors_philox) for the tests.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "cd_common.cuh"
#include "cd_internal.h"

namespace mshqc_cd {
namespace {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

// ten rounds of Philox4x32 on counter c with key (k0, k1)
__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = kPhiloxM0 * c[0], hi0 = __umulhi(kPhiloxM0, c[0]);
        const uint32_t lo1 = kPhiloxM1 * c[2], hi1 = __umulhi(kPhiloxM1, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
}

// Box-Muller pair (r cos 2 pi u2, r sin 2 pi u2) of one Philox block
__device__ __forceinline__ void std_normal_pair(uint64_t seed, uint64_t ctr, double* zc, double* zs) {
    uint32_t c[4] = {(uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((uint64_t)c[0] << 32) | c[1], b = ((uint64_t)c[2] << 32) | c[3];
    const double u1 = ((double)(a >> 11) + 0.5) * 0x1.0p-53;
    const double u2 = ((double)(b >> 11) + 0.5) * 0x1.0p-53;
    const double r = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    *zc = r * cs;
    *zs = r * sn;
}

// One 32 x 32 tile pair (row block x <= column block y) of vector Q0 + q:
// out[q][mu N + nu] and its mirror element.  256 threads, 4 rows each.
__global__ void __launch_bounds__(256) gen_vectors_kernel(uint64_t seed, const double* __restrict__ scale,
                                                          int64_t N, int64_t Q0, double* __restrict__ out) {
    __shared__ double tile[32][33];
    const int nb = (int)((N + 31) / 32);
    const int x = (int)(blockIdx.x / nb), y = (int)(blockIdx.x % nb);
    if (y < x) return;                          // the mirror tile is written by (y, x)
    const int64_t q = blockIdx.y, Q = Q0 + q;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const double s = scale[Q];
    double* o = out + q * N * N;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = ty + 8 * k;
        const int64_t mu = (int64_t)x * 32 + r, nu = (int64_t)y * 32 + tx;
        double v = 0.0;
        if (mu < N && nu < N) {
            // the pair's block sits at counter (Q N + min) N + max (x < y: mu < nu)
            const int64_t lo = mu < nu ? mu : nu, hi = mu < nu ? nu : mu;
            double z1, z2;
            std_normal_pair(seed, ((uint64_t)Q * N + lo) * N + hi, &z1, &z2);
            if (mu == nu) z2 = z1;
            v = s * (0.5 * (z1 + z2));
            o[mu * N + nu] = v;
        }
        tile[r][tx] = v;
    }
    if (x == y) return;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = ty + 8 * k;
        const int64_t nu = (int64_t)y * 32 + r, mu = (int64_t)x * 32 + tx;
        if (mu < N && nu < N) o[nu * N + mu] = tile[tx][r];
    }
}

constexpr size_t kChunkBytes = size_t(2) << 30;   // generated vectors per chunk: 2 GB

}  // namespace

int64_t vectors_chunk_size(const mshqc_cd_ctx* ctx) {
    if (!ctx->L_gen) return ctx->M;
    // MSHQC_CD_GEN_CHUNK (vectors per chunk) overrides the 2 GB default
    if (const char* env = std::getenv("MSHQC_CD_GEN_CHUNK")) {
        const long long c = std::atoll(env);
        if (c > 0) return std::min<int64_t>(ctx->M, (int64_t)c);
    }
    const int64_t per_q = ctx->N * ctx->N * (int64_t)sizeof(double);
    return std::max<int64_t>(1, std::min<int64_t>(ctx->M, (int64_t)kChunkBytes / per_q));
}

int vectors_chunk(mshqc_cd_ctx* ctx, int64_t Q0, int64_t mc, const double** out) {
    const int64_t N = ctx->N;
    if (!ctx->L_gen) {
        *out = ctx->L.as<double>() + Q0 * N * N;
        return MSHQC_CD_OK;
    }
    CD_ALLOC(ctx->Lchunk, sizeof(double) * (size_t)(mc * N * N), false);
    const int64_t nb = cdiv(N, 32);
    dim3 grid((unsigned)(nb * nb), (unsigned)mc);
    gen_vectors_kernel<<<grid, 256, 0, ctx->stream>>>(ctx->gen_seed, ctx->gen_scale.as<double>(), N, Q0,
                                                      ctx->Lchunk.as<double>());
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    *out = ctx->Lchunk.as<double>();
    return MSHQC_CD_OK;
}

}  // namespace mshqc_cd

using namespace mshqc_cd;

extern "C" MSHQC_CD_API int mshqc_cd_gen_vectors(mshqc_cd_ctx* ctx, int64_t nbf, int64_t nvec, uint64_t seed,
                                                 double sigma) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (nbf <= 0 || nvec <= 0) return set_error(MSHQC_CD_ERR_ARG, "nbf and nvec must be positive");
    if (!std::isfinite(sigma)) return set_error(MSHQC_CD_ERR_NUMERIC, "sigma is not finite");
    DeviceGuard g(ctx->device);
    ctx->invalidate_all();
    ctx->L.release();
    std::vector<double> s((size_t)nvec);
    for (int64_t q = 0; q < nvec; ++q) s[q] = std::pow(10.0, -6.0 * (double)q / (double)nvec) * sigma;
    CD_ALLOC(ctx->gen_scale, sizeof(double) * (size_t)nvec, false);
    CD_CUDA(cudaMemcpyAsync(ctx->gen_scale.p, s.data(), sizeof(double) * (size_t)nvec, cudaMemcpyHostToDevice,
                            ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->N = nbf;
    ctx->M = nvec;
    ctx->Mp = round_up(nvec, 16);
    ctx->gen_seed = seed;
    ctx->L_set = true;
    ctx->L_gen = true;
    return MSHQC_CD_OK;
}
