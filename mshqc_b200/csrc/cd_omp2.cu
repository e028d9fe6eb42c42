// CD-OMP2 on the GPU: one gradient evaluation of CholeskyOMP2::compute
// (reference src/mp2/cholesky_omp2.cc:442-466) and its orbital-rotation loop
// (:375-424, :427-512), FP64 throughout.
//
// Amplitudes: the same-spin t = ((ia|jb) - (ib|ja))/D and opposite-spin
// t = (ia|jb)/D of the reference (:94-183) are formed block by block (rows i
// of one block, every j) by an FP64 GEMM and the element-wise pass of
// amp_elem.cuh; nothing of size o^2 v^2 is ever held.  Each amplitude block
// A[(i,a)][(j,b)] feeds the one-particle density (:232-326) through two
// contractions:
//   column Gram  Gvv_x[a][b] += c * sum_i sum_(j,c) A[(i,a)][(j,c)] A[(i,b)][(j,c)]
//   row Gram     Goo_y[i][j] += c * sum_(k,a) sum_b A[(k,a)][(i,b)] A[(k,a)][(j,b)]
// Same-spin blocks give both blocks of their own spin (c = +1/2, -1/2, using
// t[i,k,a,b] = t[k,i,b,a]); the opposite-spin pass with alpha rows gives
// Gvv_alpha and Goo_beta, the one with beta rows Gvv_beta and Goo_alpha.
// The generalized Fock matrix (:331-369) uses the Cholesky J and K:
//   J = sum_Q <L^Q, P_tot> L^Q,   K_s = sum_Q L^Q P_s L^Q,
// with Z^Q = P_s L^Q for all Q as one batched GEMM and K_s as one GEMM over
// the composite index (Q, nu); F_mo = C^T (H + J - K_s) C.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "amp_elem.cuh"
#include "cd_common.cuh"
#include "cd_internal.h"
#include "gemm_f64.cuh"
#include "pair_energy_f64.cuh"

namespace mshqc_cd {
namespace {

// out[k] += alpha * sum_s parts[s * n + k], in a fixed order
__global__ void sum_parts_acc_kernel(const double* __restrict__ parts, int S, int64_t n, double alpha,
                                     double* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += parts[(int64_t)s * n + k];
    out[k] += alpha * acc;
}

// X[(c * R + r) * w + b] = A[r * ldA + c * w + b]: column blocks of width w
// become rows, so that a row Gram is an ordinary GEMM over K = (r, b)
__global__ void regroup_kernel(const double* __restrict__ A, int64_t ldA, int64_t R, int64_t nc, int64_t w,
                               double* __restrict__ X) {
    const int64_t total = R * nc * w;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t % w, rest = t / w, r = rest % R, c = rest / R;
        X[t] = A[r * ldA + c * w + b];
    }
}

// out[q] = sum_k L[q * n + k] P[k] (one CTA per q, fixed-order tree)
__global__ void dot_rows_kernel(const double* __restrict__ L, int64_t n, const double* __restrict__ P,
                                double* __restrict__ out) {
    __shared__ double red[256];
    const double* row = L + (int64_t)blockIdx.x * n;
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += 256) s = fma(row[k], P[k], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// G (N x N) = blockdiag(Goo (o x o), Gvv (v x v, row stride vp)), zero elsewhere
__global__ void blockdiag_kernel(const double* __restrict__ Goo, const double* __restrict__ Gvv, int64_t N,
                                 int64_t o, int64_t vp, double* __restrict__ G) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= N * N) return;
    const int64_t r = t / N, c = t % N;
    double x = 0.0;
    if (r < o && c < o) x = Goo[r * o + c];
    else if (r >= o && c >= o) x = Gvv[(r - o) * vp + (c - o)];
    G[t] = x;
}

// out = a + s * b (elementwise)
__global__ void axpy_kernel(const double* __restrict__ a, double s, const double* __restrict__ b, int64_t n,
                            double* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) out[t] = a[t] + s * b[t];
}

__global__ void identity_kernel(double* __restrict__ A, int64_t N) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < N * N) A[t] = (t / N == t % N) ? 1.0 : 0.0;
}

unsigned blocks_for(int64_t n, int threads = 256) { return (unsigned)cdiv(n, threads); }

// C (+)= alpha * sum_k X[m][k] X[n][k] for the o x o Gram of X (o rows of
// length K), split over K so that enough CTAs run; partials go to `ws`.
int gram_rows_splitk(mshqc_cd_ctx* ctx, const double* X, int64_t o, int64_t K, double alpha, double* C,
                     mshqc_cd::DevBuf& ws) {
    const int64_t tiles = cdiv(o, 64) * cdiv(o, 64);
    const int64_t S = std::max<int64_t>(1, std::min<int64_t>(512, cdiv(4 * ctx->num_sms, tiles)));
    const int64_t Kc = (K / S) / 16 * 16, Krem = K - S * Kc;
    CD_ALLOC(ws, sizeof(double) * (size_t)(S * o * o), false);
    GemmF64Args g{};
    g.M = (int)o;  g.N = (int)o;  g.K = (int)Kc;  g.batch = (int)S;
    g.A = X;  g.lda = K;  g.sA = Kc;
    g.B = X;  g.ldb = K;  g.sB = Kc;
    g.C = ws.as<double>();  g.ldc = o;  g.sC = o * o;
    g.alpha = 1.0;  g.beta = 0.0;
    if (Kc > 0) {
        CD_CUDA(gemm_f64(g, true, true, ctx->stream));
        ctx->launches++;
    } else {
        CD_CUDA(cudaMemsetAsync(ws.p, 0, sizeof(double) * (size_t)(S * o * o), ctx->stream));
    }
    if (Krem > 0) {
        GemmF64Args t = g;
        t.K = (int)Krem;  t.batch = 1;
        t.A = X + S * Kc;  t.B = X + S * Kc;
        t.beta = Kc > 0 ? 1.0 : 0.0;
        CD_CUDA(gemm_f64(t, true, true, ctx->stream));
        ctx->launches++;
    }
    sum_parts_acc_kernel<<<blocks_for(o * o), 256, 0, ctx->stream>>>(ws.as<double>(), (int)S, o * o, alpha, C);
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    return MSHQC_CD_OK;
}

struct OpdmOut {
    double* Goo[2];   // o_s x o_s
    double* Gvv[2];   // vp_s x vp_s (padded)
};

// One amplitude pass: rows i of spin sx (blocks), columns every j of spin sy.
// Gvv_sx += col_coef * column Gram, Goo_sy += row_coef * row Gram; tile
// energies to `partial` when it is not null.
template <int MODE>
int opdm_pass(mshqc_cd_ctx* ctx, int sx, int sy, double col_coef, double row_coef, const OpdmOut& out,
              double* partial) {
    SpinState& X = ctx->spin[sx];
    SpinState& Y = ctx->spin[sy];
    const int64_t N = ctx->N, Mp = ctx->Mp;
    const int64_t ox = X.nocc, vx = N - ox, vpx = X.vp;
    const int64_t oy = Y.nocc, vy = N - oy, vpy = Y.vp;
    const int64_t ldS = oy * vpy;
    size_t free_b = 0, total_b = 0;
    CD_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per_i = 2 * sizeof(double) * (size_t)vpx * ldS;
    const size_t budget = std::max<size_t>(per_i, std::min<size_t>(free_b / 4, size_t(24) << 30));
    const int bi = (int)std::max<int64_t>(1, std::min<int64_t>(ox, (int64_t)(budget / per_i)));
    CD_ALLOC(ctx->W, per_i / 2 * bi, false);
    CD_ALLOC(ctx->amp, per_i / 2 * bi, false);
    if (!partial) {
        // energies of this pass are not needed: throw-away slots, one per pair
        CD_ALLOC(ctx->pair_sum, sizeof(double) * (size_t)(ox * oy), false);
        partial = ctx->pair_sum.as<double>();
    }
    for (int i0 = 0; i0 < ox; i0 += bi) {
        const int nbi = (int)std::min<int64_t>(bi, ox - i0);
        const int64_t R = (int64_t)nbi * vpx;
        // S[(i,a)][(j,b)] = sum_Q X[(i,a)][Q] Y[(j,b)][Q]
        GemmF64Args g{};
        g.M = (int)R;  g.N = (int)ldS;  g.K = (int)Mp;  g.batch = 1;
        g.A = X.B64.as<double>() + (int64_t)i0 * vpx * Mp;  g.lda = Mp;  g.sA = 0;
        g.B = Y.B64.as<double>();  g.ldb = Mp;  g.sB = 0;
        g.C = ctx->W.as<double>();  g.ldc = ldS;  g.sC = 0;
        g.alpha = 1.0;  g.beta = 0.0;
        CD_CUDA(gemm_f64(g, true, true, ctx->stream));
        ctx->launches++;
        AmpElemArgs e{};
        e.S = ctx->W.as<double>();
        e.ldS = ldS;
        e.rsx = (int)vpx;  e.csy = (int)vpy;  e.ksy = (int)vpy;
        e.ox = (int)ox;  e.oy = (int)oy;  e.vx = (int)vx;  e.vy = (int)vy;
        e.i0 = i0;  e.nbi = nbi;  e.j0 = 0;  e.nbj = (int)oy;  e.wgt = 1.0;
        e.eox = X.eps.as<double>();  e.evx = e.eox + ox;
        e.eoy = Y.eps.as<double>();  e.evy = e.eoy + oy;
        e.A64 = ctx->amp.as<double>();  e.ldA = ldS;
        e.partial = partial;   // no dE/de here: prow, pcol, pocc stay null
        amp_elem_kernel<MODE, false><<<(unsigned)(nbi * oy), 256, 0, ctx->stream>>>(e);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
        // column Gram: Gvv_x[a][b] += c * sum_K A[(i,a)][K] A[(i,b)][K], one GEMM per i
        for (int ii = 0; ii < nbi; ++ii) {
            GemmF64Args h{};
            h.M = (int)vpx;  h.N = (int)vpx;  h.K = (int)ldS;  h.batch = 1;
            h.A = ctx->amp.as<double>() + (int64_t)ii * vpx * ldS;  h.lda = ldS;  h.sA = 0;
            h.B = h.A;  h.ldb = ldS;  h.sB = 0;
            h.C = out.Gvv[sx];  h.ldc = vpx;  h.sC = 0;
            h.alpha = col_coef;  h.beta = 1.0;
            CD_CUDA(gemm_f64(h, true, true, ctx->stream));
            ctx->launches++;
        }
        // row Gram: regroup the columns j of A into rows, then an o_y x o_y Gram
        regroup_kernel<<<(unsigned)std::min<int64_t>(cdiv(R * ldS, 256), (int64_t)ctx->num_sms * 32), 256, 0,
                         ctx->stream>>>(ctx->amp.as<double>(), ldS, R, oy, vpy, ctx->W.as<double>());
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
        CD_RC(gram_rows_splitk(ctx, ctx->W.as<double>(), oy, R * vpy, row_coef, out.Goo[sy], ctx->omp2_ws));
    }
    return MSHQC_CD_OK;
}

// Device layout of ctx->opdm (doubles): Goo_a, Goo_b, Gvv_a (vp_a^2), Gvv_b,
// then per spin P, F (N^2 each), then G, T, J, K, Fao (N^2 each), coef (M).
struct Omp2Buffers {
    double* Goo[2];
    double* Gvv[2];
    double* P[2];
    double* F[2];
    double *G, *T, *J, *K, *Fao, *coef, *deps;
};

int omp2_buffers(mshqc_cd_ctx* ctx, Omp2Buffers& b) {
    const int64_t N = ctx->N, M = ctx->M;
    const int64_t o0 = ctx->spin[0].nocc, o1 = ctx->spin[1].nocc;
    const int64_t vp0 = round_up(N - o0, 64), vp1 = round_up(N - o1, 64);
    const int64_t n = o0 * o0 + o1 * o1 + vp0 * vp0 + vp1 * vp1 + 9 * N * N + M + 2 * N;
    CD_ALLOC(ctx->opdm, sizeof(double) * (size_t)n, false);
    double* p = ctx->opdm.as<double>();
    b.Goo[0] = p;  p += o0 * o0;
    b.Goo[1] = p;  p += o1 * o1;
    b.Gvv[0] = p;  p += vp0 * vp0;
    b.Gvv[1] = p;  p += vp1 * vp1;
    b.P[0] = p;  p += N * N;
    b.P[1] = p;  p += N * N;
    b.F[0] = p;  p += N * N;
    b.F[1] = p;  p += N * N;
    b.G = p;  p += N * N;
    b.T = p;  p += N * N;
    b.J = p;  p += N * N;
    b.K = p;  p += N * N;
    b.Fao = p;  p += N * N;
    b.coef = p;  p += M;
    b.deps = p;
    return MSHQC_CD_OK;
}

// P = C[:, :o] C[:, :o]^T (C column-major)
int occupied_density(mshqc_cd_ctx* ctx, const double* C, int64_t o, double* P) {
    const int64_t N = ctx->N;
    GemmF64Args g{};
    g.M = (int)N;  g.N = (int)N;  g.K = (int)o;  g.batch = 1;
    g.A = C;  g.lda = N;  g.sA = 0;
    g.B = C;  g.ldb = N;  g.sB = 0;
    g.C = P;  g.ldc = N;  g.sC = 0;
    g.alpha = 1.0;  g.beta = 0.0;
    CD_CUDA(gemm_f64(g, false, false, ctx->stream));
    ctx->launches++;
    return MSHQC_CD_OK;
}

// The gradient evaluation at the context's current orbitals.  Pref[s]: the
// reference density of spin s (device, N*N).  Outputs stay in the buffers;
// *e_mp2 receives the OMP2 energy (same-spin + opposite-spin).
int omp2_pieces_device(mshqc_cd_ctx* ctx, const double* const Pref[2], Omp2Buffers& b, double* e_mp2) {
    const int64_t N = ctx->N, M = ctx->M, NN = N * N;
    for (int s = 0; s < 2; ++s) CD_RC(ensure_transform(ctx, s, MSHQC_CD_FP64));
    CD_RC(omp2_buffers(ctx, b));
    const int64_t o0 = ctx->spin[0].nocc, o1 = ctx->spin[1].nocc;
    const int64_t vp0 = ctx->spin[0].vp, vp1 = ctx->spin[1].vp;
    // OPDM blocks start at zero
    CD_CUDA(cudaMemsetAsync(b.Goo[0], 0, sizeof(double) * (size_t)(o0 * o0 + o1 * o1 + vp0 * vp0 + vp1 * vp1),
                            ctx->stream));
    CD_ALLOC(ctx->totals, sizeof(double) * 16, false);
    const int64_t n0 = o0 * o0, n1 = o1 * o1, n2 = o0 * o1;   // one energy per pair
    CD_ALLOC(ctx->partial, sizeof(double) * (size_t)(n0 + n1 + n2), false);
    double* part = ctx->partial.as<double>();
    OpdmOut out{{b.Goo[0], b.Goo[1]}, {b.Gvv[0], b.Gvv[1]}};
    begin_stage(ctx, ST_AMPLITUDE);
    CD_RC(opdm_pass<AMP_SAME_SPIN>(ctx, 0, 0, 0.5, -0.5, out, part));
    CD_RC(opdm_pass<AMP_SAME_SPIN>(ctx, 1, 1, 0.5, -0.5, out, part + n0));
    CD_RC(opdm_pass<AMP_OPPOSITE_SPIN>(ctx, 0, 1, 1.0, -1.0, out, part + n0 + n1));
    CD_RC(opdm_pass<AMP_OPPOSITE_SPIN>(ctx, 1, 0, 1.0, -1.0, out, nullptr));
    end_stage(ctx);
    const int64_t offs[3] = {0, n0, n0 + n1}, cnt[3] = {n0, n1, n2};
    for (int k = 0; k < 3; ++k) {
        reduce_total_kernel<<<1, 256, 0, ctx->stream>>>(part + offs[k], (int)cnt[k], ctx->totals.as<double>() + k);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
    }
    double e3[3] = {0.0, 0.0, 0.0};
    CD_CUDA(cudaMemcpyAsync(e3, ctx->totals.p, sizeof(e3), cudaMemcpyDeviceToHost, ctx->stream));

    begin_stage(ctx, ST_OTHER);
    // P_s = Pref_s + C_s blockdiag(Goo_s, Gvv_s) C_s^T
    for (int s = 0; s < 2; ++s) {
        const SpinState& sp = ctx->spin[s];
        const double* C = sp.C.as<double>();
        blockdiag_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(b.Goo[s], b.Gvv[s], N, sp.nocc, sp.vp, b.G);
        CD_CUDA(cudaGetLastError());
        // T = C G  (T[r][c] = sum_k C(r,k) G(k,c))
        GemmF64Args g{};
        g.M = (int)N;  g.N = (int)N;  g.K = (int)N;  g.batch = 1;
        g.A = C;  g.lda = N;  g.B = b.G;  g.ldb = N;  g.C = b.T;  g.ldc = N;
        g.alpha = 1.0;  g.beta = 0.0;
        CD_CUDA(gemm_f64(g, false, false, ctx->stream));
        // P = T C^T + Pref
        CD_CUDA(cudaMemcpyAsync(b.P[s], Pref[s], sizeof(double) * NN, cudaMemcpyDeviceToDevice, ctx->stream));
        GemmF64Args h{};
        h.M = (int)N;  h.N = (int)N;  h.K = (int)N;  h.batch = 1;
        h.A = b.T;  h.lda = N;  h.B = C;  h.ldb = N;  h.C = b.P[s];  h.ldc = N;
        h.alpha = 1.0;  h.beta = 1.0;
        CD_CUDA(gemm_f64(h, true, false, ctx->stream));
        ctx->launches += 3;
    }
    // J = sum_Q <L^Q, P_a + P_b> L^Q
    axpy_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(b.P[0], 1.0, b.P[1], NN, b.G);
    dot_rows_kernel<<<(unsigned)M, 256, 0, ctx->stream>>>(ctx->L.as<double>(), NN, b.G, b.coef);
    CD_CUDA(cudaGetLastError());
    {
        GemmF64Args g{};
        g.M = 1;  g.N = (int)NN;  g.K = (int)M;  g.batch = 1;
        g.A = b.coef;  g.lda = M;  g.B = ctx->L.as<double>();  g.ldb = NN;  g.C = b.J;  g.ldc = NN;
        g.alpha = 1.0;  g.beta = 0.0;
        CD_CUDA(gemm_f64(g, true, false, ctx->stream));
        ctx->launches += 3;
    }
    CD_ALLOC(ctx->Zt, sizeof(double) * (size_t)(M * NN), false);
    for (int s = 0; s < 2; ++s) {
        const double* C = ctx->spin[s].C.as<double>();
        // Z^Q = P_s L^Q for every Q (batched)
        GemmF64Args z{};
        z.M = (int)N;  z.N = (int)N;  z.K = (int)N;  z.batch = (int)M;
        z.A = b.P[s];  z.lda = N;  z.sA = 0;
        z.B = ctx->L.as<double>();  z.ldb = N;  z.sB = NN;
        z.C = ctx->Zt.as<double>();  z.ldc = N;  z.sC = NN;
        z.alpha = 1.0;  z.beta = 0.0;
        CD_CUDA(gemm_f64(z, true, false, ctx->stream));
        // K[mu][lam] = sum_{(Q,nu)} L^Q(mu,nu) Z^Q(nu,lam)
        GemmF64Args k{};
        k.M = (int)N;  k.N = (int)N;  k.K = (int)(M * N);  k.batch = 1;
        k.A = ctx->L.as<double>();  k.lda = N;
        k.B = ctx->Zt.as<double>();  k.ldb = N;
        k.C = b.K;  k.ldc = N;
        k.alpha = 1.0;  k.beta = 0.0;
        CD_CUDA(gemm_f64(k, false, false, ctx->stream));
        // F_ao = H + J - K
        axpy_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(ctx->Hcore.as<double>(), 1.0, b.J, NN, b.Fao);
        axpy_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(b.Fao, -1.0, b.K, NN, b.Fao);
        CD_CUDA(cudaGetLastError());
        // T = F_ao C, then F_mo (column-major): out[c][r] = sum_mu T(mu,c) C(mu,r)
        GemmF64Args t{};
        t.M = (int)N;  t.N = (int)N;  t.K = (int)N;  t.batch = 1;
        t.A = b.Fao;  t.lda = N;  t.B = C;  t.ldb = N;  t.C = b.T;  t.ldc = N;
        t.alpha = 1.0;  t.beta = 0.0;
        CD_CUDA(gemm_f64(t, true, true, ctx->stream));
        GemmF64Args f{};
        f.M = (int)N;  f.N = (int)N;  f.K = (int)N;  f.batch = 1;
        f.A = b.T;  f.lda = N;  f.B = C;  f.ldb = N;  f.C = b.F[s];  f.ldc = N;
        f.alpha = 1.0;  f.beta = 0.0;
        CD_CUDA(gemm_f64(f, false, true, ctx->stream));
        ctx->launches += 6;
    }
    end_stage(ctx);
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    *e_mp2 = e3[0] + e3[1] + e3[2];
    return MSHQC_CD_OK;
}

// exp(A) for a real N x N matrix (row-major) of 1-norm norm1, by scaling and
// squaring with a degree-18 Taylor polynomial in Horner form: with
// ||A / 2^s||_1 <= 1/2 the truncation error is below 1e-22.  E and W are work
// matrices; *result points at whichever holds exp(A).
int expm_device(mshqc_cd_ctx* ctx, const double* A, double norm1, double* E, double* W, const double** result) {
    const int64_t N = ctx->N, NN = N * N;
    int s = 0;
    while (norm1 > 0.5 && s < 60) {
        norm1 *= 0.5;
        ++s;
    }
    const double scale = std::ldexp(1.0, -s);
    identity_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(E, N);
    CD_CUDA(cudaGetLastError());
    for (int k = 18; k >= 1; --k) {
        // W = I + (scale / k) A E
        identity_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(W, N);
        GemmF64Args g{};
        g.M = (int)N;  g.N = (int)N;  g.K = (int)N;  g.batch = 1;
        g.A = A;  g.lda = N;  g.B = E;  g.ldb = N;  g.C = W;  g.ldc = N;
        g.alpha = scale / k;  g.beta = 1.0;
        CD_CUDA(gemm_f64(g, true, false, ctx->stream));
        std::swap(E, W);
        ctx->launches += 2;
    }
    for (int q = 0; q < s; ++q) {
        GemmF64Args g{};
        g.M = (int)N;  g.N = (int)N;  g.K = (int)N;  g.batch = 1;
        g.A = E;  g.lda = N;  g.B = E;  g.ldb = N;  g.C = W;  g.ldc = N;
        g.alpha = 1.0;  g.beta = 0.0;
        CD_CUDA(gemm_f64(g, true, false, ctx->stream));
        std::swap(E, W);
        ctx->launches++;
    }
    *result = E;
    return MSHQC_CD_OK;
}

// C_s <- C_s exp(-kappa), kappa from w (v x o, column-major w(a,i)) and the
// MO Fock diagonal exactly as reference src/mp2/cholesky_omp2.cc:375-400
// (damping 0.5, level shift 0.2, |denominator| >= 1e-2), then the new
// orbitals replace the context's.  F_host: F_mo column-major N x N.
int rotate_spin(mshqc_cd_ctx* ctx, int spin, const std::vector<double>& F_host) {
    const int64_t N = ctx->N, NN = N * N, o = ctx->spin[spin].nocc, v = N - o;
    std::vector<double> A(NN, 0.0);   // row-major A = -kappa
    for (int64_t a = 0; a < v; ++a)
        for (int64_t i = 0; i < o; ++i) {
            double diff = F_host[(o + a) * N + (o + a)] - F_host[i * N + i] + 0.2;
            if (std::abs(diff) < 1e-2) diff = diff >= 0 ? 1e-2 : -1e-2;
            const double w = 2.0 * F_host[i * N + (o + a)];   // w(a,i) = 2 F(o+a, i)
            const double val = (w / diff) * 0.5;
            A[(o + a) * N + i] = -val;    // -kappa(o+a, i)
            A[i * N + (o + a)] = val;     // -kappa(i, o+a)
        }
    double norm1 = 0.0;
    for (int64_t c = 0; c < N; ++c) {
        double col = 0.0;
        for (int64_t r = 0; r < N; ++r) col += std::abs(A[r * N + c]);
        norm1 = std::max(norm1, col);
    }
    CD_ALLOC(ctx->omp2_ws, sizeof(double) * (size_t)(4 * NN), false);
    double* dA = ctx->omp2_ws.as<double>();
    double* E0 = dA + NN;
    double* E1 = E0 + NN;
    double* Cn = E1 + NN;
    CD_CUDA(cudaMemcpyAsync(dA, A.data(), sizeof(double) * NN, cudaMemcpyHostToDevice, ctx->stream));
    const double* E = nullptr;
    CD_RC(expm_device(ctx, dA, norm1, E0, E1, &E));
    // column-major C_new = C E: as row-major arrays C_new^T = E^T C^T
    double* C = ctx->spin[spin].C.as<double>();
    GemmF64Args g{};
    g.M = (int)N;  g.N = (int)N;  g.K = (int)N;  g.batch = 1;
    g.A = E;  g.lda = N;  g.B = C;  g.ldb = N;  g.C = Cn;  g.ldc = N;
    g.alpha = 1.0;  g.beta = 0.0;
    CD_CUDA(gemm_f64(g, false, false, ctx->stream));
    ctx->launches++;
    CD_CUDA(cudaMemcpyAsync(C, Cn, sizeof(double) * NN, cudaMemcpyDeviceToDevice, ctx->stream));
    return invalidate_spin(ctx, spin);
}

int require_omp2_inputs(mshqc_cd_ctx* ctx) {
    if (!ctx->L_set) return set_error(MSHQC_CD_ERR_STATE, "Cholesky vectors not set");
    if (!ctx->spin[0].set || !ctx->spin[1].set)
        return set_error(MSHQC_CD_ERR_STATE, "OMP2 needs alpha and beta orbitals (set both; equal for RHF)");
    if (!ctx->H_set) return set_error(MSHQC_CD_ERR_STATE, "core Hamiltonian not set");
    if (ctx->L_gen)
        return set_error(MSHQC_CD_ERR_UNSUPPORTED,
                         "OMP2 needs stored Cholesky vectors (mshqc_cd_set_vectors), not generated ones");
    return MSHQC_CD_OK;
}

// reference densities: caller's (host or device) or C_occ C_occ^T
int reference_densities(mshqc_cd_ctx* ctx, const double* Pa, const double* Pb, int where, double* dst[2]) {
    const int64_t N = ctx->N, NN = N * N;
    const double* in[2] = {Pa, Pb};
    for (int s = 0; s < 2; ++s) {
        if (in[s]) {
            if (where == MSHQC_CD_HOST)
                CD_RC(upload(ctx, dst[s], in[s], sizeof(double) * NN));
            else
                CD_CUDA(cudaMemcpyAsync(dst[s], in[s], sizeof(double) * NN, cudaMemcpyDeviceToDevice,
                                        ctx->stream));
        } else {
            CD_RC(occupied_density(ctx, ctx->spin[s].C.as<double>(), ctx->spin[s].nocc, dst[s]));
        }
    }
    return MSHQC_CD_OK;
}

// norm2[q] = sum_k L[q * n + k]^2 (one CTA per q, fixed-order tree)
__global__ void row_norm2_kernel(const double* __restrict__ L, int64_t n, double* __restrict__ norm2) {
    __shared__ double red[256];
    const double* row = L + (int64_t)blockIdx.x * n;
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += 256) s = fma(row[k], row[k], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) norm2[blockIdx.x] = red[0];
}

// Z^q = 0 for the vectors whose Frobenius norm is at most `thr` (the
// exchange screening of src/scf/cholesky_rhf.cc:120-126); norm2[q] = |L^q|^2
__global__ void screen_slabs_kernel(double* __restrict__ Z, const double* __restrict__ norm2, int64_t nn,
                                    double thr) {
    if (norm2[blockIdx.y] > thr * thr) return;
    double* z = Z + (int64_t)blockIdx.y * nn;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nn; t += (int64_t)gridDim.x * blockDim.x)
        z[t] = 0.0;
}

// Cholesky Coulomb and exchange matrices of the SCF Fock builds,
//   J = sum_Q <L^Q, P_tot> L^Q,   K_s = sum_Q L^Q P_s L^Q,
// P_tot = P[0] (nspin 1) or P[0] + P[1] (nspin 2), over chunks of vectors
// (stored or generated): per chunk the coefficients <L^Q, P_tot> (one dot
// product per vector), J += coef . L as one GEMM, Z^Q = P_s L^Q as one batched
// GEMM and K_s += L . Z as one GEMM over the composite index (Q, nu).  All
// matrices are N x N and symmetric; device pointers on the context stream.
int cholesky_jk_device(mshqc_cd_ctx* ctx, int nspin, const double* const P[2], bool screen, double* J,
                       double* const K[2], double* work) {
    const int64_t N = ctx->N, NN = N * N, M = ctx->M;
    const double* Ptot = P[0];
    if (nspin == 2) {
        axpy_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(P[0], 1.0, P[1], NN, work);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
        Ptot = work;
    }
    CD_CUDA(cudaMemsetAsync(J, 0, sizeof(double) * NN, ctx->stream));
    for (int s = 0; s < nspin; ++s) CD_CUDA(cudaMemsetAsync(K[s], 0, sizeof(double) * NN, ctx->stream));
    // vectors per chunk: the generator's chunk, and at most 2 GB of Z
    const int64_t mc_max = std::max<int64_t>(
        1, std::min<int64_t>({vectors_chunk_size(ctx), (int64_t)((size_t(2) << 30) / (sizeof(double) * NN)),
                              (int64_t)65535}));
    CD_ALLOC(ctx->Zt, sizeof(double) * (size_t)(mc_max * NN), false);
    CD_ALLOC(ctx->omp2_ws, sizeof(double) * (size_t)(2 * mc_max), false);
    double* coef = ctx->omp2_ws.as<double>();
    double* norm2 = coef + mc_max;
    for (int64_t Q0 = 0; Q0 < M; Q0 += mc_max) {
        const int64_t mc = std::min<int64_t>(mc_max, M - Q0);
        const double* Lc = nullptr;
        CD_RC(vectors_chunk(ctx, Q0, mc, &Lc));
        dot_rows_kernel<<<(unsigned)mc, 256, 0, ctx->stream>>>(Lc, NN, Ptot, coef);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
        GemmF64Args g{};
        g.M = 1;  g.N = (int)NN;  g.K = (int)mc;  g.batch = 1;
        g.A = coef;  g.lda = mc;  g.B = Lc;  g.ldb = NN;  g.C = J;  g.ldc = NN;
        g.alpha = 1.0;  g.beta = 1.0;
        CD_CUDA(gemm_f64(g, true, false, ctx->stream));
        ctx->launches++;
        if (screen) {
            row_norm2_kernel<<<(unsigned)mc, 256, 0, ctx->stream>>>(Lc, NN, norm2);
            CD_CUDA(cudaGetLastError());
            ctx->launches++;
        }
        for (int s = 0; s < nspin; ++s) {
            GemmF64Args z{};
            z.M = (int)N;  z.N = (int)N;  z.K = (int)N;  z.batch = (int)mc;
            z.A = P[s];  z.lda = N;  z.sA = 0;
            z.B = Lc;  z.ldb = N;  z.sB = NN;
            z.C = ctx->Zt.as<double>();  z.ldc = N;  z.sC = NN;
            z.alpha = 1.0;  z.beta = 0.0;
            CD_CUDA(gemm_f64(z, true, false, ctx->stream));
            ctx->launches++;
            if (screen) {
                dim3 grid((unsigned)std::min<int64_t>(cdiv(NN, 256), 1024), (unsigned)mc);
                screen_slabs_kernel<<<grid, 256, 0, ctx->stream>>>(ctx->Zt.as<double>(), norm2, NN, 1e-8);
                CD_CUDA(cudaGetLastError());
                ctx->launches++;
            }
            GemmF64Args k{};
            k.M = (int)N;  k.N = (int)N;  k.K = (int)(mc * N);  k.batch = 1;
            k.A = Lc;  k.lda = N;
            k.B = ctx->Zt.as<double>();  k.ldb = N;
            k.C = K[s];  k.ldc = N;
            k.alpha = 1.0;  k.beta = 1.0;
            CD_CUDA(gemm_f64(k, false, false, ctx->stream));
            ctx->launches++;
        }
    }
    return MSHQC_CD_OK;
}

}  // namespace
}  // namespace mshqc_cd

using namespace mshqc_cd;

extern "C" {

MSHQC_CD_API int mshqc_cd_set_core_hamiltonian(mshqc_cd_ctx* ctx, const double* H, int where) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (!H) return set_error(MSHQC_CD_ERR_ARG, "H is null");
    if (!ctx->L_set) return set_error(MSHQC_CD_ERR_STATE, "set_vectors must precede set_core_hamiltonian");
    DeviceGuard g(ctx->device);
    const int64_t NN = ctx->N * ctx->N;
    CD_ALLOC(ctx->Hcore, sizeof(double) * (size_t)NN, false);
    if (where == MSHQC_CD_HOST) {
        CD_RC(upload(ctx, ctx->Hcore.p, H, sizeof(double) * NN));
    } else {
        CD_CUDA(cudaMemcpyAsync(ctx->Hcore.p, H, sizeof(double) * NN, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CD_RC(check_finite_device(ctx, ctx->Hcore.as<double>(), NN, "H"));
    ctx->H_set = true;
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}

MSHQC_CD_API int mshqc_cd_get_orbitals(mshqc_cd_ctx* ctx, int spin, double* C, int where) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (spin != MSHQC_CD_ALPHA && spin != MSHQC_CD_BETA)
        return set_error(MSHQC_CD_ERR_ARG, "spin must be 0 (alpha) or 1 (beta)");
    if (!ctx->spin[spin].set) return set_error(MSHQC_CD_ERR_STATE, "orbitals of this spin not set");
    DeviceGuard g(ctx->device);
    CD_RC(download(ctx, C, ctx->spin[spin].C.p, sizeof(double) * ctx->N * ctx->N, where));
    return MSHQC_CD_OK;
}

MSHQC_CD_API int mshqc_cd_omp2_pieces(mshqc_cd_ctx* ctx, const double* P_a, const double* P_b, double* e_mp2,
                                      double* Goo_a, double* Gvv_a, double* Goo_b, double* Gvv_b, double* F_a,
                                      double* F_b, int where) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    CD_RC(require_omp2_inputs(ctx));
    DeviceGuard g(ctx->device);
    reset_stages(ctx);
    const int64_t N = ctx->N, NN = N * N;
    // reference densities (ctx->scratch is not used by the FP64 passes)
    CD_ALLOC(ctx->scratch, sizeof(double) * (size_t)(2 * NN), false);
    double* pr[2] = {ctx->scratch.as<double>(), ctx->scratch.as<double>() + NN};
    CD_RC(reference_densities(ctx, P_a, P_b, where, pr));
    Omp2Buffers b{};
    double e = 0.0;
    const double* prc[2] = {pr[0], pr[1]};
    CD_RC(omp2_pieces_device(ctx, prc, b, &e));
    collect_stages(ctx);
    if (e_mp2) *e_mp2 = e;
    // OPDM blocks out without the padding
    for (int s = 0; s < 2; ++s) {
        const int64_t o = ctx->spin[s].nocc, v = N - o, vp = ctx->spin[s].vp;
        double* goo = s == 0 ? Goo_a : Goo_b;
        double* gvv = s == 0 ? Gvv_a : Gvv_b;
        double* f = s == 0 ? F_a : F_b;
        if (goo) CD_RC(download(ctx, goo, b.Goo[s], sizeof(double) * o * o, where));
        if (gvv) {
            if (where == MSHQC_CD_HOST) {
                std::vector<double> tmp((size_t)(vp * vp));
                CD_RC(download(ctx, tmp.data(), b.Gvv[s], sizeof(double) * vp * vp, MSHQC_CD_HOST));
                for (int64_t a = 0; a < v; ++a)
                    std::memcpy(gvv + a * v, tmp.data() + a * vp, sizeof(double) * v);
            } else {
                CD_CUDA(cudaMemcpy2DAsync(gvv, sizeof(double) * v, b.Gvv[s], sizeof(double) * vp,
                                          sizeof(double) * v, v, cudaMemcpyDeviceToDevice, ctx->stream));
                CD_CUDA(cudaStreamSynchronize(ctx->stream));
            }
        }
        if (f) CD_RC(download(ctx, f, b.F[s], sizeof(double) * NN, where));
    }
    return MSHQC_CD_OK;
}

MSHQC_CD_API int mshqc_cd_omp2(mshqc_cd_ctx* ctx, const mshqc_cd_omp2_config* cfg, const double* P_a,
                               const double* P_b, int where, mshqc_cd_omp2_result* res) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (!cfg || !res) return set_error(MSHQC_CD_ERR_ARG, "cfg and res must be non-null");
    if (cfg->max_iterations < 0) return set_error(MSHQC_CD_ERR_ARG, "max_iterations must be >= 0");
    CD_RC(require_omp2_inputs(ctx));
    DeviceGuard g(ctx->device);
    const int64_t N = ctx->N, NN = N * N;
    const int64_t na = ctx->spin[0].nocc, nb = ctx->spin[1].nocc;
    std::memset(res, 0, sizeof(*res));
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1];
    CD_CUDA(cudaEventRecord(e0, ctx->stream));
    reset_stages(ctx);
    // reference densities live in ctx->scratch for the whole loop
    CD_ALLOC(ctx->scratch, sizeof(double) * (size_t)(2 * NN), false);
    double* pref[2] = {ctx->scratch.as<double>(), ctx->scratch.as<double>() + NN};
    CD_RC(reference_densities(ctx, P_a, P_b, where, pref));
    const double* prc[2] = {pref[0], pref[1]};
    double e_prev = cfg->e_scf, e_corr = 0.0;
    int iter = 0, converged = 0;
    std::vector<double> Fa((size_t)NN), Fb((size_t)NN);
    while (iter < cfg->max_iterations) {
        ++iter;
        Omp2Buffers b{};
        CD_RC(omp2_pieces_device(ctx, prc, b, &e_corr));
        CD_CUDA(cudaMemcpyAsync(Fa.data(), b.F[0], sizeof(double) * NN, cudaMemcpyDeviceToHost, ctx->stream));
        CD_CUDA(cudaMemcpyAsync(Fb.data(), b.F[1], sizeof(double) * NN, cudaMemcpyDeviceToHost, ctx->stream));
        CD_CUDA(cudaStreamSynchronize(ctx->stream));
        const double e_cur = cfg->e_scf + e_corr;
        double g2 = 0.0;
        for (int s = 0; s < 2; ++s) {
            const std::vector<double>& F = s == 0 ? Fa : Fb;
            const int64_t o = s == 0 ? na : nb;
            for (int64_t i = 0; i < o; ++i)
                for (int64_t a = o; a < N; ++a) {
                    const double w = 2.0 * F[i * N + a];
                    g2 += w * w;
                }
        }
        const double g_norm = std::sqrt(g2);
        if (g_norm < cfg->gradient_threshold && std::abs(e_cur - e_prev) < cfg->energy_threshold) {
            converged = 1;
            break;
        }
        CD_RC(rotate_spin(ctx, 0, Fa));
        CD_RC(occupied_density(ctx, ctx->spin[0].C.as<double>(), na, pref[0]));
        if (na != nb) {
            CD_RC(rotate_spin(ctx, 1, Fb));
            CD_RC(occupied_density(ctx, ctx->spin[1].C.as<double>(), nb, pref[1]));
        } else {
            // closed-shell count: beta follows alpha (reference :481-484)
            CD_CUDA(cudaMemcpyAsync(ctx->spin[1].C.p, ctx->spin[0].C.p, sizeof(double) * NN,
                                    cudaMemcpyDeviceToDevice, ctx->stream));
            CD_RC(invalidate_spin(ctx, 1));
            CD_CUDA(cudaMemcpyAsync(pref[1], pref[0], sizeof(double) * NN, cudaMemcpyDeviceToDevice,
                                    ctx->stream));
        }
        e_prev = e_cur;
    }
    CD_CUDA(cudaEventRecord(e1, ctx->stream));
    CD_CUDA(cudaEventSynchronize(e1));
    collect_stages(ctx);
    float ms = 0.0f;
    CD_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    res->energy_scf = cfg->e_scf;
    res->energy_mp2_corr = e_corr;
    res->energy_total = e_prev;   // the reference reports the previous iterate's total
    res->iterations = iter;
    res->converged = converged;
    res->ms_total = ms;
    return MSHQC_CD_OK;
}

MSHQC_CD_API int mshqc_cd_cholesky_fock(mshqc_cd_ctx* ctx, int nspin, const double* P_a, const double* P_b,
                                        const double* H, int screen_exchange, double* F_a, double* F_b,
                                        double* J, double* K_a, double* K_b, int where) {
    if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");
    if (nspin != 1 && nspin != 2) return set_error(MSHQC_CD_ERR_ARG, "nspin must be 1 (RHF) or 2 (UHF)");
    if (!P_a || (nspin == 2 && !P_b)) return set_error(MSHQC_CD_ERR_ARG, "density missing");
    if ((F_a || (nspin == 2 && F_b)) && !H) return set_error(MSHQC_CD_ERR_ARG, "a Fock matrix needs H");
    if (where != MSHQC_CD_HOST && where != MSHQC_CD_DEVICE) return set_error(MSHQC_CD_ERR_ARG, "bad where");
    if (!ctx->L_set) return set_error(MSHQC_CD_ERR_STATE, "set_vectors (or gen_vectors) must come first");
    DeviceGuard g(ctx->device);
    reset_stages(ctx);
    const int64_t NN = ctx->N * ctx->N;
    // P_a P_b H | J K_a K_b | F work
    CD_ALLOC(ctx->opdm, sizeof(double) * (size_t)(8 * NN), false);
    double* base = ctx->opdm.as<double>();
    double* P[2] = {base, base + NN};
    double* Hd = base + 2 * NN;
    double* Jd = base + 3 * NN;
    double* Kd[2] = {base + 4 * NN, base + 5 * NN};
    double* Fd = base + 6 * NN;
    double* work = base + 7 * NN;
    const double* in[3] = {P_a, nspin == 2 ? P_b : nullptr, H};
    double* dst[3] = {P[0], P[1], Hd};
    for (int k = 0; k < 3; ++k) {
        if (!in[k]) continue;
        if (where == MSHQC_CD_HOST)
            CD_RC(upload(ctx, dst[k], in[k], sizeof(double) * NN));
        else
            CD_CUDA(cudaMemcpyAsync(dst[k], in[k], sizeof(double) * NN, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    const double* Pc[2] = {P[0], P[1]};
    begin_stage(ctx, ST_OTHER);
    CD_RC(cholesky_jk_device(ctx, nspin, Pc, nspin == 1 && screen_exchange != 0, Jd, Kd, work));
    end_stage(ctx);
    if (J) CD_RC(download(ctx, J, Jd, sizeof(double) * NN, where));
    double* Kout[2] = {K_a, K_b};
    double* Fout[2] = {F_a, F_b};
    // RHF (src/scf/cholesky_rhf.cc:136): F = H + J - K/2 with the total density;
    // UHF (src/scf/cholesky_uhf.cc:90-98): F_s = H + J - K_s
    const double kf = nspin == 1 ? -0.5 : -1.0;
    for (int s = 0; s < nspin; ++s) {
        if (Kout[s]) CD_RC(download(ctx, Kout[s], Kd[s], sizeof(double) * NN, where));
        if (Fout[s]) {
            axpy_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(Hd, 1.0, Jd, NN, Fd);
            axpy_kernel<<<blocks_for(NN), 256, 0, ctx->stream>>>(Fd, kf, Kd[s], NN, Fd);
            CD_CUDA(cudaGetLastError());
            ctx->launches += 2;
            CD_RC(download(ctx, Fout[s], Fd, sizeof(double) * NN, where));
        }
    }
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    collect_stages(ctx);
    return MSHQC_CD_OK;
}

}  // extern "C"
