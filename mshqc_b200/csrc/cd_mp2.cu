// Orchestration of the Cholesky-MP2 kernels: half transforms, pair energies,
// reductions.  Called from the C ABI (cd_abi.cu) with the device selected.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cd_common.cuh"
#include "cd_internal.h"
#include "gemm_f64.cuh"
#include "pair_energy_f64.cuh"
#include "pair_energy_tc.cuh"
#include "split_bf16.cuh"
#include "gamma_tc.cuh"
#include "vtile_tc.cuh"
#include "amp_elem.cuh"
#include "ozaki_i8.cuh"

namespace mshqc_cd {


namespace {

// out[k] = alpha * sum_s parts[s * n + k], in a fixed order
__global__ void sum_partials_kernel(const double* __restrict__ parts, int S, int64_t n, double alpha,
                                    double* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += parts[(int64_t)s * n + k];
    out[k] = alpha * acc;
}

// Partitioned backward: whether the next unit (block pair, or occupied block
// of an FP64 pass) belongs to this context's share.  Units beyond the plan
// (which a mismatch between plan_partition and the passes would produce)
// belong to nobody; run_gradient checks the count afterwards.
bool owns_next(mshqc_cd_ctx* ctx) {
    const int64_t k = ctx->part_next++;
    if (!ctx->part_active) return true;
    return k < (int64_t)ctx->part_owned.size() && ctx->part_owned[(size_t)k] != 0;
}

// ---------------------------------------------------------------------------
// occupied block sizes of the backward passes
// ---------------------------------------------------------------------------
// Unpartitioned, a block is as large as a share of the free device memory
// allows (fewer, larger launches).  Partitioned, the block sizes are a
// function of the problem dimensions and the number of ranks only, so that
// every rank enumerates the same units whatever memory its GPU has free: at
// most the staging these fixed budgets hold, and small enough that there are
// about 32 units per rank for the cost-balanced plan (4 per rank in the
// opposite-spin passes, whose units are blocks of rows against all columns).
// MSHQC_CD_BWD_BLOCK (occupied orbitals per block) overrides both rules in
// every pass.
constexpr size_t kPartTcBudget = size_t(16) << 30;
constexpr size_t kPartF64Budget = size_t(8) << 30;

// Wave pacing of the persistent tile kernels (WavePacer in sm100_ptx.cuh):
// copies per epoch and epochs of slack.  On by default for Gamma (its K runs
// to 57600 and unpaced CTAs drift apart: 7x the DRAM traffic), off for the
// integral tiles (K = M; pacing them changed nothing at N=2000).
// MSHQC_CD_PACE (Gamma) and MSHQC_CD_PACE_TILES (integral tiles) = off
// disables it, = <every>,<slack> enables it with those values.
void pace_params(int* every, int* slack, const char* var, bool on_by_default) {
    *every = on_by_default ? 16 : 0;
    *slack = 2;
    const char* env = std::getenv(var);
    if (!env) return;
    if (std::strcmp(env, "off") == 0) {
        *every = 0;
        return;
    }
    int e = 0, s = 0;
    if (std::sscanf(env, "%d,%d", &e, &s) == 2 && e > 0 && s >= 0) {
        *every = e;
        *slack = s;
    }
}

int64_t env_block() {
    const char* env = std::getenv("MSHQC_CD_BWD_BLOCK");
    if (!env) return 0;
    const long long b = std::atoll(env);
    return b > 0 ? (int64_t)b : 0;
}

// block sizes (rows bI, columns bJ) of a tensor-core pass; staging per (i, j)
// of S (FP32, VS columns) and the four BF16 amplitude operands
void tc_block_sizes(const mshqc_cd_ctx* ctx, int64_t ox, int64_t oy, int64_t VRx, int64_t VRy, int64_t VSy,
                    bool sym, size_t free_budget, int64_t* bI, int64_t* bJ) {
    const bool part = ctx->part_active;
    const size_t budget = part ? kPartTcBudget : free_budget;
    if (sym) {
        const double per_b2 = (double)VRx * (4.0 * VSy + 8.0 * VRy);
        *bI = std::max<int64_t>(1, std::min<int64_t>(ox, (int64_t)std::sqrt((double)budget / per_b2)));
        if (part) {
            // nb blocks give nb (nb + 1) / 2 block pairs: about 32 per rank
            const int64_t nb = (int64_t)std::ceil(std::sqrt(64.0 * ctx->part_size));
            *bI = std::min<int64_t>(*bI, std::max<int64_t>(1, cdiv(ox, nb)));
        }
    } else {
        const double per_i = (double)VRx * oy * (4.0 * VSy + 8.0 * VRy);
        *bI = std::max<int64_t>(1, std::min<int64_t>(ox, (int64_t)((double)budget / per_i)));
        if (part) *bI = std::min<int64_t>(*bI, std::max<int64_t>(1, cdiv(ox, 4 * (int64_t)ctx->part_size)));
    }
    if (const int64_t b = env_block()) *bI = std::min<int64_t>(ox, b);
    *bJ = sym ? *bI : oy;
}

// block sizes (rows bI, columns bJ) of an FP64 pass: staging of S and of the
// amplitudes, both FP64, per (i, j)
void f64_block_sizes(const mshqc_cd_ctx* ctx, int64_t ox, int64_t oy, int64_t vpx, int64_t vpy, bool sym,
                     size_t free_budget, int64_t* bI, int64_t* bJ) {
    const bool part = ctx->part_active;
    const double budget = (double)(part ? kPartF64Budget : free_budget);
    const double per_ij = 2.0 * sizeof(double) * (double)vpx * (double)vpy;
    if (sym) {
        *bI = std::max<int64_t>(1, std::min<int64_t>(ox, (int64_t)std::sqrt(budget / per_ij)));
        if (part) {
            const int64_t nb = (int64_t)std::ceil(std::sqrt(64.0 * ctx->part_size));
            *bI = std::min<int64_t>(*bI, std::max<int64_t>(1, cdiv(ox, nb)));
        }
    } else {
        *bI = std::max<int64_t>(1, std::min<int64_t>(ox, (int64_t)(budget / (per_ij * oy))));
        if (part) *bI = std::min<int64_t>(*bI, std::max<int64_t>(1, cdiv(ox, 4 * (int64_t)ctx->part_size)));
    }
    if (const int64_t b = env_block()) *bI = std::min<int64_t>(ox, b);
    *bJ = sym ? *bI : oy;
}

int require_inputs(mshqc_cd_ctx* ctx, int spin) {
    if (!ctx->L_set) return set_error(MSHQC_CD_ERR_STATE, "Cholesky vectors not set");
    if (!ctx->spin[spin].set)
        return set_error(MSHQC_CD_ERR_STATE,
                         spin == 0 ? "alpha orbitals not set" : "beta orbitals not set");
    return MSHQC_CD_OK;
}

// ---------------------------------------------------------------------------
// transforms shared over occupied orbitals (partition + host collectives)
// ---------------------------------------------------------------------------
// Rank r of R owns the occupied orbitals [r p, min(o, (r + 1) p)),
// p = ceil(o / R); per-orbital buffers (B, Gamma) then hold R p rows so that
// every rank's chunk has the same size for the collectives.
bool sharded(const mshqc_cd_ctx* ctx) { return ctx->part_active && ctx->coll_set && ctx->part_size > 1; }
int64_t shard_p(const mshqc_cd_ctx* ctx, int64_t o) { return cdiv(o, ctx->part_size); }
void shard_range(const mshqc_cd_ctx* ctx, int64_t o, int64_t* lo, int64_t* hi) {
    if (!sharded(ctx)) {
        *lo = 0;
        *hi = o;
        return;
    }
    const int64_t p = shard_p(ctx, o);
    *lo = std::min(o, (int64_t)ctx->part_rank * p);
    *hi = std::min(o, *lo + p);
}
int64_t b_rows(const mshqc_cd_ctx* ctx, int64_t o) { return sharded(ctx) ? shard_p(ctx, o) * ctx->part_size : o; }

int run_collective(mshqc_cd_ctx* ctx, bool gather, double* buf, int64_t count) {
    int (*fn)(double*, int64_t, void*, void*) = gather ? ctx->coll.allgather : ctx->coll.reduce_scatter;
    const int rc = fn(buf, count, (void*)ctx->stream, ctx->coll.user);
    if (rc != 0)
        return set_error(MSHQC_CD_ERR_STATE, std::string(gather ? "allgather" : "reduce_scatter") +
                                                 " callback failed with " + std::to_string(rc));
    return MSHQC_CD_OK;
}

// FP64 half transform of one spin into the padded [i][a][Q] layout, for the
// occupied orbitals [lo, hi) (Y holds rows i - lo; B rows outside stay zero).
int transform_f64(mshqc_cd_ctx* ctx, int spin, int64_t lo, int64_t hi) {
    SpinState& s = ctx->spin[spin];
    const int64_t N = ctx->N, M = ctx->M, Mp = ctx->Mp, o = s.nocc, v = N - o, ni = hi - lo;
    const int64_t vp = round_up(v, 64);
    CD_ALLOC(ctx->Y, sizeof(double) * (size_t)std::max<int64_t>(1, ni) * M * N, false);
    CD_ALLOC(s.B64, sizeof(double) * (size_t)b_rows(ctx, o) * vp * Mp, true);
    s.vp = vp;
    ctx->Y_spin = spin;
    ctx->Y_lo = lo;
    ctx->Y_hi = hi;
    s.B64_valid = true;
    s.B64_prec = MSHQC_CD_FP64;
    if (ni <= 0) return MSHQC_CD_OK;
    const double* C = s.C.as<double>();
    // Y[i][(Q,nu)] = sum_mu C[mu,i] L[Q][nu*N + mu], one chunk of Q at a time
    const int64_t qc = vectors_chunk_size(ctx);
    for (int64_t Q0 = 0; Q0 < M; Q0 += qc) {
        const int64_t mc = std::min(qc, M - Q0);
        const double* Lc = nullptr;
        CD_RC(vectors_chunk(ctx, Q0, mc, &Lc));
        GemmF64Args g1{};
        g1.M = (int)ni;
        g1.N = (int)(mc * N);
        g1.K = (int)N;
        g1.batch = 1;
        g1.A = C + lo * N;  g1.lda = N;  g1.sA = 0;
        g1.B = Lc;  g1.ldb = N;  g1.sB = 0;
        g1.C = ctx->Y.as<double>() + Q0 * N;  g1.ldc = M * N;  g1.sC = 0;
        g1.alpha = 1.0;  g1.beta = 0.0;
        CD_CUDA(gemm_f64(g1, true, true, ctx->stream));
        ctx->launches++;
    }
    // B[i][a][Q] = sum_nu C[nu, o+a] Y[i][Q][nu]
    GemmF64Args g2{};
    g2.M = (int)v;
    g2.N = (int)M;
    g2.K = (int)N;
    g2.batch = (int)ni;
    g2.A = C + o * N;  g2.lda = N;  g2.sA = 0;
    g2.B = ctx->Y.as<double>();  g2.ldb = N;  g2.sB = M * N;
    g2.C = s.B64.as<double>() + lo * vp * Mp;  g2.ldc = Mp;  g2.sC = vp * Mp;
    g2.alpha = 1.0;  g2.beta = 0.0;
    CD_CUDA(gemm_f64(g2, true, true, ctx->stream));
    ctx->launches++;
    return MSHQC_CD_OK;
}

// Bytes of int8 slices one product operand may hold (bounds the vectors
// sub-chunks of the first product and the orbital batches of the second).
constexpr size_t kSliceBytes = size_t(2) << 30;

bool int8_transform_enabled(const mshqc_cd_ctx* ctx) {
    if (ctx->N > ozaki::kMaxK) return false;
    const char* env = std::getenv("MSHQC_CD_TRANSFORM");
    return !(env && std::strcmp(env, "f64") == 0);
}

// The forward half transform of a mixed request runs on the int8 tensor
// cores from N = 512 on; below, the FP64 DMMA products are faster (forward
// transform of the gradient step, one box: N=400 1.8 ms FP64 vs 2.6 ms int8,
// N=600 8.8 vs 7.6 ms) and their B is exact.  The transposed transforms keep
// the int8 products at every size (N=400: 3.4 vs 6.8 ms).
// MSHQC_CD_TRANSFORM=i8 forces the int8 products, =f64 the FP64 ones.
constexpr int64_t kInt8ForwardMinN = 512;
bool int8_forward_enabled(const mshqc_cd_ctx* ctx) {
    if (!int8_transform_enabled(ctx)) return false;
    const char* env = std::getenv("MSHQC_CD_TRANSFORM");
    if (env && std::strcmp(env, "i8") == 0) return true;
    return ctx->N >= kInt8ForwardMinN;
}

// The same half transform as transform_f64 with both products on the int8
// tensor cores (ozaki_i8.cuh): Y = C_occ^T L per vectors chunk, then
// B_i = C_vir^T Y_i^T in batches of occupied orbitals.  Accuracy of the
// slices (about 2^-33 of the row maxima per term), not FP64 rounding: used by
// the mixed-precision path only.
int transform_i8(mshqc_cd_ctx* ctx, int spin, int64_t lo, int64_t hi) {
    using namespace ozaki;
    SpinState& s = ctx->spin[spin];
    const int64_t N = ctx->N, M = ctx->M, Mp = ctx->Mp, o = s.nocc, v = N - o, ni = hi - lo;
    const int64_t vp = round_up(v, 64);
    CD_ALLOC(ctx->Y, sizeof(double) * (size_t)std::max<int64_t>(1, ni) * M * N, false);
    CD_ALLOC(s.B64, sizeof(double) * (size_t)b_rows(ctx, o) * vp * Mp, true);
    CD_ALLOC(ctx->oz_flag, sizeof(int) * 2, true);
    s.vp = vp;
    ctx->Y_spin = spin;
    ctx->Y_lo = lo;
    ctx->Y_hi = hi;
    s.B64_valid = true;
    s.B64_prec = MSHQC_CD_FP16X3;
    if (ni <= 0) return MSHQC_CD_OK;
    int* err = ctx->oz_flag.as<int>();
    const double* C = s.C.as<double>();
    // rows of C^T: occupied orbitals of the slice (first product), virtual orbitals (second)
    OzakiOperand Ao = ozaki_operand(ni, N, BM, 1), Av = ozaki_operand(v, N, BM, 1);
    const size_t ao_bytes = operand_bytes(Ao.Rp, Ao.Kp);
    CD_ALLOC(ctx->oz_a, ao_bytes + operand_bytes(Av.Rp, Av.Kp), false);
    CD_ALLOC(ctx->oz_ea, sizeof(int) * (size_t)(Ao.Rp + Av.Rp), false);
    Ao.q = ctx->oz_a.as<int8_t>();  Ao.e = ctx->oz_ea.as<int>();
    Av.q = Ao.q + ao_bytes;         Av.e = Ao.e + Ao.Rp;
    CD_CUDA(ozaki_slice(C + lo * N, N, 0, Ao, ctx->num_sms, ctx->stream));
    CD_CUDA(ozaki_slice(C + o * N, N, 0, Av, ctx->num_sms, ctx->stream));
    ctx->launches += 2;
    // Y[i][(Q,nu)] = sum_mu C[mu,i] L[Q][nu*N + mu]
    const int64_t per_q = (int64_t)operand_bytes(padded_rows(N, BN), padded_k(N));
    const int64_t qs = std::max<int64_t>(1, (int64_t)kSliceBytes / per_q);
    const int64_t qc = vectors_chunk_size(ctx);
    for (int64_t Q0 = 0; Q0 < M; Q0 += qc) {
        const int64_t mc = std::min(qc, M - Q0);
        const double* Lc = nullptr;
        CD_RC(vectors_chunk(ctx, Q0, mc, &Lc));
        for (int64_t q0 = 0; q0 < mc; q0 += qs) {
            const int64_t ms = std::min(qs, mc - q0);
            OzakiOperand Bl = ozaki_operand(ms * N, N, BN, 1);
            CD_ALLOC(ctx->oz_b, operand_bytes(Bl.Rp, Bl.Kp), false);
            CD_ALLOC(ctx->oz_eb, sizeof(int) * (size_t)Bl.Rp, false);
            Bl.q = ctx->oz_b.as<int8_t>();  Bl.e = ctx->oz_eb.as<int>();
            CD_CUDA(ozaki_slice(Lc + q0 * N * N, N, 0, Bl, ctx->num_sms, ctx->stream));
            CD_CUDA(ozaki_gemm(Ao, true, Bl, false, ctx->Y.as<double>() + (Q0 + q0) * N, M * N, 0, 1.0, 0.0, err,
                               ctx->num_sms, ctx->stream));
            ctx->launches += 2;
        }
    }
    // B[i][a][Q] = sum_nu C[nu, o+a] Y[i][Q][nu], a batch of orbitals i at a time
    const int64_t per_i = (int64_t)operand_bytes(padded_rows(M, BN), padded_k(N));
    const int64_t ib = std::max<int64_t>(1, std::min<int64_t>(ni, (int64_t)kSliceBytes / per_i));
    for (int64_t i0 = lo; i0 < hi; i0 += ib) {
        const int64_t nb = std::min(ib, hi - i0);
        OzakiOperand By = ozaki_operand(M, N, BN, (int)nb);
        CD_ALLOC(ctx->oz_b, operand_bytes(By.Rp, By.Kp) * (size_t)nb, false);
        CD_ALLOC(ctx->oz_eb, sizeof(int) * (size_t)(By.Rp * nb), false);
        By.q = ctx->oz_b.as<int8_t>();  By.e = ctx->oz_eb.as<int>();
        CD_CUDA(ozaki_slice(ctx->Y.as<double>() + (i0 - lo) * M * N, N, M * N, By, ctx->num_sms, ctx->stream));
        CD_CUDA(ozaki_gemm(Av, true, By, false, s.B64.as<double>() + i0 * vp * Mp, Mp, vp * Mp, 1.0, 0.0, err,
                           ctx->num_sms, ctx->stream));
        ctx->launches += 2;
    }
    int herr = 0;
    CD_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    if (herr)
        return set_error(MSHQC_CD_ERR_TIMEOUT, "int8 tensor-core transform gave up waiting (site " +
                                                   std::to_string(herr) + ")");
    return MSHQC_CD_OK;
}

struct UnitTables {
    std::vector<int2> pairs, blocks;
};

UnitTables make_tables(int mode, int ox, int oy, int nbx, int nby) {
    UnitTables t;
    if (mode == PAIR_OPPOSITE_SPIN) {
        for (int i = 0; i < ox; ++i)
            for (int j = 0; j < oy; ++j) t.pairs.push_back(make_int2(i, j));
        for (int x = 0; x < nbx; ++x)
            for (int y = 0; y < nby; y += 2) t.blocks.push_back(make_int2(x, y));
    } else {
        for (int i = 0; i < ox; ++i)
            for (int j = (mode == PAIR_RESTRICTED ? i : i + 1); j < ox; ++j)
                t.pairs.push_back(make_int2(i, j));
        for (int x = 0; x < nbx; ++x)
            for (int y = x; y < nbx; ++y) t.blocks.push_back(make_int2(x, y));
    }
    return t;
}

// Deterministic reductions of per-unit partials into pair energies and totals,
// and the host copy of the ordered pair-energy matrix.
int reduce_and_collect(mshqc_cd_ctx* ctx, int mode, const UnitTables& t, int64_t units, int npairs,
                       int nblocks, int ox, int oy, double* total, std::vector<double>& pair_mat,
                       double* total_os) {
    ctx->launches += 2;
    reduce_pairs_kernel<<<(unsigned)cdiv(npairs, 128), 128, 0, ctx->stream>>>(
        ctx->partial.as<double>(), npairs, nblocks, ctx->pair_sum.as<double>());
    CD_CUDA(cudaGetLastError());
    reduce_total_kernel<<<1, 256, 0, ctx->stream>>>(ctx->pair_sum.as<double>(), npairs,
                                                   ctx->totals.as<double>());
    CD_CUDA(cudaGetLastError());
    if (mode == PAIR_RESTRICTED && total_os) {
        ctx->launches += 2;
        reduce_pairs_kernel<<<(unsigned)cdiv(npairs, 128), 128, 0, ctx->stream>>>(
            ctx->partial.as<double>() + units, npairs, nblocks, ctx->pair_sum.as<double>() + npairs);
        CD_CUDA(cudaGetLastError());
        reduce_total_kernel<<<1, 256, 0, ctx->stream>>>(ctx->pair_sum.as<double>() + npairs, npairs,
                                                       ctx->totals.as<double>() + 1);
        CD_CUDA(cudaGetLastError());
        CD_CUDA(cudaMemcpyAsync(total_os, ctx->totals.as<double>() + 1, sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
    }
    std::vector<double> ps(npairs);
    CD_CUDA(cudaMemcpyAsync(ps.data(), ctx->pair_sum.p, sizeof(double) * npairs,
                            cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaMemcpyAsync(total, ctx->totals.p, sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int p = 0; p < npairs; ++p) {
        const int i = t.pairs[p].x, j = t.pairs[p].y;
        if (mode == PAIR_OPPOSITE_SPIN) {
            pair_mat[(size_t)i * oy + j] = ps[p];
        } else if (i == j) {
            pair_mat[(size_t)i * ox + j] = ps[p];
        } else {
            pair_mat[(size_t)i * ox + j] = 0.5 * ps[p];
            pair_mat[(size_t)j * ox + i] = 0.5 * ps[p];
        }
    }
    return MSHQC_CD_OK;
}

// One FP64 pair-energy pass.  Returns the total in *total and fills the
// ordered pair-energy matrix (row-major ox*oy) in pair_mat.
int pair_pass_f64(mshqc_cd_ctx* ctx, int mode, int sx, int sy, double* total,
                  std::vector<double>& pair_mat, double* total_os = nullptr) {
    const SpinState& X = ctx->spin[sx];
    const SpinState& Y = ctx->spin[sy];
    const int ox = (int)X.nocc, oy = (int)Y.nocc;
    const int vx = (int)(ctx->N - ox), vy = (int)(ctx->N - oy);
    const int nbx = (int)(X.vp / 64), nby = (int)(Y.vp / 64);
    UnitTables t = make_tables(mode, ox, oy, nbx, nby);
    const int npairs = (int)t.pairs.size(), nblocks = (int)t.blocks.size();
    pair_mat.assign((size_t)ox * oy, 0.0);
    *total = 0.0;
    if (npairs == 0 || nblocks == 0) return MSHQC_CD_OK;

    const size_t tbytes = sizeof(int2) * (t.pairs.size() + t.blocks.size());
    CD_ALLOC(ctx->tables, tbytes, false);
    int2* dpairs = ctx->tables.as<int2>();
    int2* dblocks = dpairs + npairs;
    CD_CUDA(cudaMemcpyAsync(dpairs, t.pairs.data(), sizeof(int2) * npairs, cudaMemcpyHostToDevice,
                            ctx->stream));
    CD_CUDA(cudaMemcpyAsync(dblocks, t.blocks.data(), sizeof(int2) * nblocks,
                            cudaMemcpyHostToDevice, ctx->stream));
    const int64_t units = (int64_t)npairs * nblocks;
    CD_ALLOC(ctx->partial, sizeof(double) * units * 2, false);
    CD_ALLOC(ctx->pair_sum, sizeof(double) * npairs * 2, false);
    CD_ALLOC(ctx->totals, sizeof(double) * 8, false);

    PairF64Args a{};
    a.X = X.B64.as<double>();
    a.Y = Y.B64.as<double>();
    a.vx = vx;  a.vy = vy;
    a.vpx = (int)X.vp;  a.vpy = (int)Y.vp;
    a.Mp = (int)ctx->Mp;
    a.eox = X.eps.as<double>();  a.evx = a.eox + ox;
    a.eoy = Y.eps.as<double>();  a.evy = a.eoy + oy;
    a.pairs = dpairs;
    a.blocks = dblocks;
    a.nblocks = nblocks;
    a.partial = ctx->partial.as<double>();
    a.partial2 = ctx->partial.as<double>() + units;
    const size_t smem = pair_f64_detail::SMEM_BYTES;
    begin_stage(ctx, ST_PAIR);
    if (mode == PAIR_RESTRICTED) {
        CD_CUDA(cudaFuncSetAttribute(pair_energy_f64_kernel<PAIR_RESTRICTED>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        pair_energy_f64_kernel<PAIR_RESTRICTED><<<(unsigned)units, 256, smem, ctx->stream>>>(a);
    } else if (mode == PAIR_SAME_SPIN) {
        CD_CUDA(cudaFuncSetAttribute(pair_energy_f64_kernel<PAIR_SAME_SPIN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        pair_energy_f64_kernel<PAIR_SAME_SPIN><<<(unsigned)units, 256, smem, ctx->stream>>>(a);
    } else {
        CD_CUDA(cudaFuncSetAttribute(pair_energy_f64_kernel<PAIR_OPPOSITE_SPIN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        pair_energy_f64_kernel<PAIR_OPPOSITE_SPIN><<<(unsigned)units, 256, smem, ctx->stream>>>(a);
    }
    end_stage(ctx);
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    CD_RC(reduce_and_collect(ctx, mode, t, units, npairs, nblocks, ox, oy, total, pair_mat, total_os));
    return MSHQC_CD_OK;
}


// ---------------------------------------------------------------------------
// FP16x3 tensor-core path
// ---------------------------------------------------------------------------
int64_t tc_rows(int64_t v) { return 128 * round_up(cdiv(v, 128), 2); }

// fixed-point hi/lo split of one spin's FP64 MO vectors into the blocked layout,
// with the per-row exponents, exact diagonal integrals and hi/lo row norms
int split_fixed(mshqc_cd_ctx* ctx, int spin, int layout) {
    SpinState& s = ctx->spin[spin];
    const int64_t o = s.nocc, v = ctx->N - s.nocc, M = ctx->M, Mp = ctx->Mp;
    const int64_t rows = tc_rows(v), nqc = Mp / 16;
    const size_t n = (size_t)o * nqc * rows * 16;
    const bool pair_layout = layout == 1;
    CD_ALLOC(s.Bhi, (pair_layout ? 2 : 1) * n * sizeof(uint16_t), false);
    if (!pair_layout) CD_ALLOC(s.Blo, n * sizeof(uint16_t), false);
    CD_ALLOC(s.expo, sizeof(int) * o * rows, true);
    CD_ALLOC(s.diag, sizeof(double) * o * rows, true);
    CD_ALLOC(s.norms, sizeof(double) * 2 * o * rows, true);
    s.vp16 = rows;
    s.Mp16 = Mp;
    double* nh = s.norms.as<double>();
    double* nl = nh + o * rows;
    {
        const int64_t warps = o * rows;
        const int blocks = (int)std::min<int64_t>(cdiv(warps * 32, 256), (int64_t)ctx->num_sms * 32);
        row_scale_kernel<<<blocks, 256, 0, ctx->stream>>>(
            s.B64.as<double>(), s.vp, Mp, (int)v, (int)M, o, rows, s.expo.as<int>(),
            s.diag.as<double>(), nh, nl, nullptr, 0, 0, 0, nullptr);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
    }
    {
        const int64_t threads = o * nqc * rows * 2;
        const int blocks = (int)std::min<int64_t>(cdiv(threads, 256), (int64_t)ctx->num_sms * 16);
        split_fixed_blocked_kernel<<<blocks, 256, 0, ctx->stream>>>(
            s.B64.as<double>(), s.vp, Mp, (int)v, (int)M, o, nqc, rows, s.expo.as<int>(),
            s.Bhi.as<uint16_t>(), pair_layout ? nullptr : s.Blo.as<uint16_t>(), pair_layout);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
    }
    // largest row norms: the Cauchy-Schwarz bound of the integer accumulators
    std::vector<double> hn(2 * o * rows);
    CD_CUDA(cudaMemcpyAsync(hn.data(), nh, sizeof(double) * 2 * o * rows, cudaMemcpyDeviceToHost,
                            ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    s.max_norm_hi = s.max_norm_lo = 0.0;
    for (int64_t r = 0; r < o * rows; ++r) {
        s.max_norm_hi = std::max(s.max_norm_hi, hn[r]);
        s.max_norm_lo = std::max(s.max_norm_lo, hn[o * rows + r]);
    }
    s.B16_valid = true;
    s.B16_layout = layout;
    return MSHQC_CD_OK;
}

// exact sum_Q B_alpha[i][a][Q] B_beta[i][a][Q] for the opposite-spin diagonal
int opposite_spin_diag(mshqc_cd_ctx* ctx) {
    if (ctx->diag_os_valid) return MSHQC_CD_OK;
    SpinState& A = ctx->spin[0];
    SpinState& B = ctx->spin[1];
    const int64_t oa = A.nocc, va = ctx->N - A.nocc, rows = A.vp16;
    const int o2 = (int)std::min(A.nocc, B.nocc);
    const int v2 = (int)std::min(ctx->N - A.nocc, ctx->N - B.nocc);
    CD_ALLOC(ctx->diag_os, sizeof(double) * std::max<int64_t>(1, (int64_t)o2 * rows), true);
    CD_ALLOC(ctx->scratch, sizeof(double) * (size_t)(oa * rows * 4), false);
    double* tmp = ctx->scratch.as<double>();
    int* etmp = reinterpret_cast<int*>(tmp + 3 * oa * rows);
    const int64_t warps = oa * rows;
    const int blocks = (int)std::min<int64_t>(cdiv(warps * 32, 256), (int64_t)ctx->num_sms * 32);
    row_scale_kernel<<<blocks, 256, 0, ctx->stream>>>(
        A.B64.as<double>(), A.vp, ctx->Mp, (int)va, (int)ctx->M, oa, rows, etmp, tmp,
        tmp + oa * rows, tmp + 2 * oa * rows, B.B64.as<double>(), B.vp, o2, v2,
        ctx->diag_os.as<double>());
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    ctx->diag_os_valid = true;
    return MSHQC_CD_OK;
}

UnitTables make_tables_tc(int mode, int ox, int oy, int nbx, int nby) {
    UnitTables t;
    if (mode == PAIR_OPPOSITE_SPIN) {
        for (int i = 0; i < ox; ++i)
            for (int j = 0; j < oy; ++j) t.pairs.push_back(make_int2(i, j));
        for (int x = 0; x < nbx; ++x)
            for (int y = 0; y < nby; y += 2) t.blocks.push_back(make_int2(x, y));
    } else {
        for (int i = 0; i < ox; ++i)
            for (int j = (mode == PAIR_RESTRICTED ? i : i + 1); j < ox; ++j)
                t.pairs.push_back(make_int2(i, j));
        for (int x = 0; x < nbx; ++x)
            for (int y = x; y < nbx; ++y) t.blocks.push_back(make_int2(x, y));
    }
    return t;
}

template <int MODE>
cudaError_t launch_tc(const PairTcArgs& a, int grid, cudaStream_t st) {
    const size_t smem = pair_tc::SMEM_BYTES;
    cudaError_t e = cudaFuncSetAttribute(pair_energy_tc_kernel<MODE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    pair_energy_tc_kernel<MODE><<<grid, pair_tc::THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

int pair_pass_tc(mshqc_cd_ctx* ctx, int mode, int sx, int sy, double* total,
                 std::vector<double>& pair_mat, double* total_os = nullptr) {
    const SpinState& X = ctx->spin[sx];
    const SpinState& Y = ctx->spin[sy];
    const int ox = (int)X.nocc, oy = (int)Y.nocc;
    const int vx = (int)(ctx->N - ox), vy = (int)(ctx->N - oy);
    const int nbx = (int)cdiv(vx, 128), nby = (int)cdiv(vy, 128);
    UnitTables t = make_tables_tc(mode, ox, oy, nbx, nby);
    const int npairs = (int)t.pairs.size(), nblocks = (int)t.blocks.size();
    pair_mat.assign((size_t)ox * oy, 0.0);
    *total = 0.0;
    if (total_os) *total_os = 0.0;
    if (npairs == 0 || nblocks == 0) return MSHQC_CD_OK;
    const size_t tbytes = sizeof(int2) * (t.pairs.size() + t.blocks.size());
    CD_ALLOC(ctx->tables, tbytes, false);
    int2* dpairs = ctx->tables.as<int2>();
    int2* dblocks = dpairs + npairs;
    CD_CUDA(cudaMemcpyAsync(dpairs, t.pairs.data(), sizeof(int2) * npairs, cudaMemcpyHostToDevice,
                            ctx->stream));
    CD_CUDA(cudaMemcpyAsync(dblocks, t.blocks.data(), sizeof(int2) * nblocks,
                            cudaMemcpyHostToDevice, ctx->stream));
    const int64_t units = (int64_t)npairs * nblocks;
    CD_ALLOC(ctx->partial, sizeof(double) * units * 2, false);
    CD_ALLOC(ctx->pair_sum, sizeof(double) * npairs * 2, false);
    CD_ALLOC(ctx->totals, sizeof(double) * 8, false);
    CD_ALLOC(ctx->flag, sizeof(int) * 4, true);

    // the integer accumulators are exact when every partial sum stays below
    // 2^24: |sum hi hi'| <= sqrt(max sum hi^2 * max sum hi'^2), likewise for
    // the cross terms (Cauchy-Schwarz over the Q index)
    {
        const double lim = 16777216.0;
        const double bhh = std::sqrt(X.max_norm_hi * Y.max_norm_hi);
        const double bx = std::sqrt(X.max_norm_hi * Y.max_norm_lo) + std::sqrt(X.max_norm_lo * Y.max_norm_hi);
        if (!(bhh < lim && bx < lim)) ctx->fixed_point_exact = 0;
    }
    if (mode == PAIR_OPPOSITE_SPIN) {
        begin_stage(ctx, ST_SPLIT);
        CD_RC(opposite_spin_diag(ctx));
        end_stage(ctx);
    }
    if (X.B16_layout != 1 || Y.B16_layout != 1)
        return set_error(MSHQC_CD_ERR_STATE, "fixed-point operands not in the pair layout");
    PairTcArgs a{};
    a.Xp = X.Bhi.as<uint16_t>();
    a.Yp = Y.Bhi.as<uint16_t>();
    a.ex = X.expo.as<int>();  a.ey = Y.expo.as<int>();
    if (mode == PAIR_OPPOSITE_SPIN) {
        a.diag = ctx->diag_os.as<double>();
        a.diag_o = (int)std::min(X.nocc, Y.nocc);
        a.diag_v = std::min(vx, vy);
    } else {
        a.diag = X.diag.as<double>();
        a.diag_o = ox;
        a.diag_v = vx;
    }
    a.rows_x = (int)X.vp16;  a.rows_y = (int)Y.vp16;
    a.nqc = (int)(ctx->Mp / 16);
    a.vx = vx;  a.vy = vy;
    a.eox = X.eps.as<double>();  a.evx = a.eox + ox;
    a.eoy = Y.eps.as<double>();  a.evy = a.eoy + oy;
    a.pairs = dpairs;  a.blocks = dblocks;  a.nblocks = nblocks;
    a.units = units;
    a.partial = ctx->partial.as<double>();
    a.partial2 = ctx->partial.as<double>() + units;
    a.err = ctx->flag.as<int>();
    const int grid = (int)std::min<int64_t>(units, ctx->num_sms);
    cudaError_t e;
    begin_stage(ctx, ST_PAIR);
    if (mode == PAIR_RESTRICTED)
        e = launch_tc<PAIR_RESTRICTED>(a, grid, ctx->stream);
    else if (mode == PAIR_SAME_SPIN)
        e = launch_tc<PAIR_SAME_SPIN>(a, grid, ctx->stream);
    else
        e = launch_tc<PAIR_OPPOSITE_SPIN>(a, grid, ctx->stream);
    end_stage(ctx);
    if (e != cudaSuccess) return cuda_error(e, "pair_energy_tc_kernel launch");
    ctx->launches++;
    int herr = 0;
    CD_CUDA(cudaMemcpyAsync(&herr, ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CD_RC(reduce_and_collect(ctx, mode, t, units, npairs, nblocks, ox, oy, total, pair_mat, total_os));
    if (herr)
        return set_error(MSHQC_CD_ERR_TIMEOUT,
                         "tensor-core pair kernel gave up waiting (site " + std::to_string(herr) + ")");
    return MSHQC_CD_OK;
}

}  // namespace

int invalidate_spin(mshqc_cd_ctx* ctx, int spin) {
    ctx->spin[spin].invalidate();
    ctx->diag_os_valid = false;
    if (ctx->Y_spin == spin) ctx->Y_spin = -1;
    return MSHQC_CD_OK;
}

int ensure_transform(mshqc_cd_ctx* ctx, int spin, int precision, int layout) {
    CD_RC(require_inputs(ctx, spin));
    SpinState& s = ctx->spin[spin];
    if (precision != MSHQC_CD_FP64 && precision != MSHQC_CD_FP16X3)
        return set_error(MSHQC_CD_ERR_ARG, "unknown precision");
    // an FP64 request never reuses int8-slice products; a mixed one reuses either
    if (!s.B64_valid || (precision == MSHQC_CD_FP64 && s.B64_prec != MSHQC_CD_FP64)) {
        begin_stage(ctx, ST_TRANSFORM);
        // shared over ranks: this rank's orbitals, then the gather of all
        int64_t lo = 0, hi = s.nocc;
        shard_range(ctx, s.nocc, &lo, &hi);
        if (precision == MSHQC_CD_FP16X3 && int8_forward_enabled(ctx))
            CD_RC(transform_i8(ctx, spin, lo, hi));
        else
            CD_RC(transform_f64(ctx, spin, lo, hi));
        if (sharded(ctx))
            CD_RC(run_collective(ctx, true, s.B64.as<double>(), shard_p(ctx, s.nocc) * s.vp * ctx->Mp));
        end_stage(ctx);
        s.B16_valid = false;
    }
    if (precision == MSHQC_CD_FP16X3 && (!s.B16_valid || s.B16_layout != layout)) {
        begin_stage(ctx, ST_SPLIT);
        CD_RC(split_fixed(ctx, spin, layout));
        end_stage(ctx);
    }
    return MSHQC_CD_OK;
}

int run_energy(mshqc_cd_ctx* ctx, int kind, int precision, mshqc_cd_energy* out) {
    std::memset(out, 0, sizeof(*out));
    ctx->fixed_point_exact = 1;
    reset_stages(ctx);
    auto pass = [&](int mode, int sx, int sy, double* tot, std::vector<double>& pm,
                    double* tot_os) {
        return precision == MSHQC_CD_FP16X3 ? pair_pass_tc(ctx, mode, sx, sy, tot, pm, tot_os)
                                            : pair_pass_f64(ctx, mode, sx, sy, tot, pm, tot_os);
    };
    CD_RC(require_inputs(ctx, 0));
    if (kind == MSHQC_CD_UNRESTRICTED) CD_RC(require_inputs(ctx, 1));
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    CD_CUDA(cudaEventRecord(e0, ctx->stream));
    CD_RC(ensure_transform(ctx, 0, precision, 1));
    if (kind == MSHQC_CD_UNRESTRICTED) CD_RC(ensure_transform(ctx, 1, precision, 1));
    CD_CUDA(cudaEventRecord(e1, ctx->stream));
    for (auto& p : ctx->pair_energy) p.clear();
    if (kind == MSHQC_CD_RESTRICTED) {
        double e_os = 0.0, e_tot = 0.0;
        CD_RC(pass(PAIR_RESTRICTED, 0, 0, &e_tot, ctx->pair_energy[0], &e_os));
        out->total = e_tot;
        out->os = e_os;
        out->ss_aa = out->ss_bb = 0.5 * (e_tot - e_os);
    } else {
        double ss_a = 0, ss_b = 0, os = 0;
        CD_RC(pass(PAIR_SAME_SPIN, 0, 0, &ss_a, ctx->pair_energy[0], nullptr));
        CD_RC(pass(PAIR_SAME_SPIN, 1, 1, &ss_b, ctx->pair_energy[1], nullptr));
        CD_RC(pass(PAIR_OPPOSITE_SPIN, 0, 1, &os, ctx->pair_energy[2], nullptr));
        out->ss_aa = ss_a;
        out->ss_bb = ss_b;
        out->os = os;
        out->total = ss_a + ss_b + os;
    }
    CD_CUDA(cudaEventRecord(e2, ctx->stream));
    CD_CUDA(cudaEventSynchronize(e2));
    collect_stages(ctx);
    float t01 = 0, t12 = 0;
    CD_CUDA(cudaEventElapsedTime(&t01, e0, e1));
    CD_CUDA(cudaEventElapsedTime(&t12, e1, e2));
    out->ms_transform = t01;
    out->ms_energy = t12;
    out->ms_total = t01 + t12;
    return MSHQC_CD_OK;
}

// ---------------------------------------------------------------------------
// backward
// ---------------------------------------------------------------------------
namespace {

// dE/dC of one spin from Gamma (ctx->gam[spin], [o][vp][Mp] FP64) with
// dE/dB = scale * Gamma (4 restricted, 2 unrestricted):
// dC[nu, o+a] = sum_{i,Q} dE/dB[i][a][Q] Y[i][Q][nu],
// dC[mu, i]   = sum_{Q,nu} L[Q][nu][mu] sum_a dE/dB[i][a][Q] C[nu, o+a].
// The transforms shared over ranks: rank r's Gamma rows [lo, hi) are
// completed by the reduce-scatter, and its transposed transforms cover those
// orbitals only (dC's other occupied columns zero); unshared: [0, o).
// Makes sure the buffer Y holds the half-transformed vectors of [lo, hi).
int transposed_prepare(mshqc_cd_ctx* ctx, int spin, bool i8, int64_t* lo, int64_t* hi, double* dC) {
    SpinState& s = ctx->spin[spin];
    shard_range(ctx, s.nocc, lo, hi);
    if (sharded(ctx))
        CD_RC(run_collective(ctx, false, ctx->gam[spin].as<double>(), shard_p(ctx, s.nocc) * s.vp * ctx->Mp));
    if (ctx->Y_spin != spin || ctx->Y_lo != *lo || ctx->Y_hi != *hi) {
        // recomputing Y rewrites B as well; shared, only this rank's rows of it
        if (i8)
            CD_RC(transform_i8(ctx, spin, *lo, *hi));
        else
            CD_RC(transform_f64(ctx, spin, *lo, *hi));
        if (sharded(ctx)) s.B64_valid = false;
    }
    if (*hi - *lo < s.nocc) CD_CUDA(cudaMemsetAsync(dC, 0, sizeof(double) * (size_t)(s.nocc * ctx->N), ctx->stream));
    if (*hi <= *lo)
        CD_CUDA(cudaMemsetAsync(dC + s.nocc * ctx->N, 0, sizeof(double) * (size_t)((ctx->N - s.nocc) * ctx->N),
                                ctx->stream));
    return MSHQC_CD_OK;
}

int transposed_transforms(mshqc_cd_ctx* ctx, int spin, double scale, double* dC) {
    SpinState& s = ctx->spin[spin];
    const int64_t N = ctx->N, M = ctx->M, Mp = ctx->Mp, o = s.nocc, v = N - o, vp = s.vp;
    // Y[i][Q][nu] (half-transformed vectors of this spin) is needed
    int64_t lo = 0, hi = o;
    CD_RC(transposed_prepare(ctx, spin, false, &lo, &hi, dC));
    const int64_t ni = hi - lo;
    if (ni <= 0) return MSHQC_CD_OK;
    const double* C = s.C.as<double>();
    const double* Gm = ctx->gam[spin].as<double>();
    // dC[nu, o+a] = scale sum_{i,Q} Gamma[i][a][Q] Y[i][Q][nu]   (row-major [a][nu] == column-major dC)
    for (int64_t i = lo; i < hi; ++i) {
        GemmF64Args g{};
        g.M = (int)v;  g.N = (int)N;  g.K = (int)M;  g.batch = 1;
        g.A = Gm + i * vp * Mp;  g.lda = Mp;  g.sA = 0;
        g.B = ctx->Y.as<double>() + (i - lo) * M * N;  g.ldb = N;  g.sB = 0;
        g.C = dC + o * N;  g.ldc = N;  g.sC = 0;
        g.alpha = scale;  g.beta = i == lo ? 0.0 : 1.0;
        CD_CUDA(gemm_f64(g, true, false, ctx->stream));
        ctx->launches++;
    }
    // W[i][Q][nu] = sum_a Gamma[i][a][Q] C[nu, o+a]   (into the Y buffer)
    {
        GemmF64Args g{};
        g.M = (int)M;  g.N = (int)N;  g.K = (int)v;  g.batch = (int)ni;
        g.A = Gm + lo * vp * Mp;  g.lda = Mp;  g.sA = vp * Mp;
        g.B = C + o * N;  g.ldb = N;  g.sB = 0;
        g.C = ctx->Y.as<double>();  g.ldc = N;  g.sC = M * N;
        g.alpha = 1.0;  g.beta = 0.0;
        CD_CUDA(gemm_f64(g, false, false, ctx->stream));
        ctx->launches++;
        ctx->Y_spin = -1;
    }
    // dC[mu, i] = scale sum_{(Q,nu)} W[i][(Q,nu)] L[(Q,nu)][mu]
    if (ctx->L_gen) {
        // generated vectors: one GEMM per chunk of Q, accumulated in order
        const int64_t qc = vectors_chunk_size(ctx);
        for (int64_t Q0 = 0; Q0 < M; Q0 += qc) {
            const int64_t mc = std::min(qc, M - Q0);
            const double* Lc = nullptr;
            CD_RC(vectors_chunk(ctx, Q0, mc, &Lc));
            GemmF64Args g{};
            g.M = (int)ni;  g.N = (int)N;  g.K = (int)(mc * N);  g.batch = 1;
            g.A = ctx->Y.as<double>() + Q0 * N;  g.lda = M * N;  g.sA = 0;
            g.B = Lc;  g.ldb = N;  g.sB = 0;
            g.C = dC + lo * N;  g.ldc = N;  g.sC = 0;
            g.alpha = scale;  g.beta = Q0 == 0 ? 0.0 : 1.0;
            CD_CUDA(gemm_f64(g, true, false, ctx->stream));
            ctx->launches++;
        }
        return MSHQC_CD_OK;
    }
    // stored vectors: only o rows, so the long K = M*N is split over S
    // independent partial products (batched GEMM) that a deterministic
    // reduction adds up
    {
        const int64_t K = M * N;
        const int64_t tiles = cdiv(ni, 64) * cdiv(N, 64);
        const int64_t S = std::max<int64_t>(1, std::min<int64_t>(256, cdiv(4 * ctx->num_sms, tiles)));
        const int64_t Kc = (K / S) / 16 * 16, Krem = K - S * Kc;   // even chunks keep 16-byte copies
        CD_ALLOC(ctx->W, sizeof(double) * (size_t)(S * ni * N), false);
        GemmF64Args g{};
        g.M = (int)ni;  g.N = (int)N;  g.K = (int)Kc;  g.batch = (int)S;
        g.A = ctx->Y.as<double>();  g.lda = M * N;  g.sA = Kc;
        g.B = ctx->L.as<double>();  g.ldb = N;  g.sB = Kc * N;
        g.C = ctx->W.as<double>();  g.ldc = N;  g.sC = ni * N;
        g.alpha = 1.0;  g.beta = 0.0;
        CD_CUDA(gemm_f64(g, true, false, ctx->stream));
        ctx->launches++;
        if (Krem > 0) {
            GemmF64Args t = g;
            t.K = (int)Krem;  t.batch = 1;
            t.A = ctx->Y.as<double>() + S * Kc;
            t.B = ctx->L.as<double>() + S * Kc * N;
            t.beta = 1.0;
            CD_CUDA(gemm_f64(t, true, false, ctx->stream));
            ctx->launches++;
        }
        sum_partials_kernel<<<(unsigned)cdiv(ni * N, 256), 256, 0, ctx->stream>>>(
            ctx->W.as<double>(), (int)S, ni * N, scale, dC + lo * N);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
    }
    return MSHQC_CD_OK;
}

// out[k] = (accumulate ? out[k] : 0) + alpha * sum_b parts[b * n + k], b in order
__global__ void sum_batches_kernel(const double* __restrict__ parts, int nb, int64_t n, double alpha,
                                   int accumulate, double* __restrict__ out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    double acc = 0.0;
    for (int b = 0; b < nb; ++b) acc += parts[(int64_t)b * n + k];
    out[k] = accumulate ? out[k] + alpha * acc : alpha * acc;
}

int sum_batches(mshqc_cd_ctx* ctx, const double* parts, int nb, int64_t n, double alpha, bool accumulate,
                double* out) {
    sum_batches_kernel<<<(unsigned)cdiv(n, 256), 256, 0, ctx->stream>>>(parts, nb, n, alpha, accumulate ? 1 : 0,
                                                                         out);
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    return MSHQC_CD_OK;
}

// The transposed transforms of the mixed path on the int8 tensor cores
// (ozaki_i8.cuh), batched so that every product has K = M, v or N:
//   dC[nu, o+a] = scale sum_i (Gamma_i Y_i)[a][nu]        batches of i, partials summed in order
//   W_i[Q][nu]  = sum_a Gamma_i[a][Q] C[nu, o+a]           batches of i, C_vir shared
//   dC[mu, i]   = scale sum_Q (W_Q L_Q)[i][mu]             batches of Q per vectors chunk
// with W_Q[i][nu] = W[i][Q][nu] and L_Q[mu][nu] = L[Q][nu][mu].
int transposed_transforms_i8(mshqc_cd_ctx* ctx, int spin, double scale, double* dC) {
    using namespace ozaki;
    SpinState& s = ctx->spin[spin];
    const int64_t N = ctx->N, M = ctx->M, Mp = ctx->Mp, o = s.nocc, v = N - o;
    int64_t lo = 0, hi = o;
    CD_RC(transposed_prepare(ctx, spin, true, &lo, &hi, dC));
    const int64_t ni = hi - lo;
    if (ni <= 0) return MSHQC_CD_OK;
    const int64_t vp = s.vp;
    const double* C = s.C.as<double>();
    const double* Gm = ctx->gam[spin].as<double>();
    double* Y = ctx->Y.as<double>();
    CD_ALLOC(ctx->oz_flag, sizeof(int) * 2, true);
    int* err = ctx->oz_flag.as<int>();
    // dC[nu, o+a]: A = Gamma_i (rows a, K = Q), B = Y_i^T (rows nu, K = Q, strided by N)
    {
        const size_t pa = operand_bytes(padded_rows(v, BM), padded_k(M));
        const size_t pb = operand_bytes(padded_rows(N, BN), padded_k(M));
        const size_t pp = sizeof(double) * (size_t)(v * N);
        const int64_t ib = std::max<int64_t>(1, std::min<int64_t>(ni, (int64_t)(2 * kSliceBytes / (pa + pb + pp))));
        CD_ALLOC(ctx->oz_a, pa * ib, false);
        CD_ALLOC(ctx->oz_b, pb * ib, false);
        CD_ALLOC(ctx->oz_p, pp * ib, false);
        CD_ALLOC(ctx->oz_ea, sizeof(int) * (size_t)(padded_rows(v, BM) * ib), false);
        CD_ALLOC(ctx->oz_eb, sizeof(int) * (size_t)(padded_rows(N, BN) * ib), false);
        for (int64_t i0 = lo; i0 < hi; i0 += ib) {
            const int64_t nb = std::min(ib, hi - i0);
            OzakiOperand A = ozaki_operand(v, M, BM, (int)nb), B = ozaki_operand(N, M, BN, (int)nb);
            A.q = ctx->oz_a.as<int8_t>();  A.e = ctx->oz_ea.as<int>();
            B.q = ctx->oz_b.as<int8_t>();  B.e = ctx->oz_eb.as<int>();
            CD_CUDA(ozaki_slice(Gm + i0 * vp * Mp, Mp, vp * Mp, A, ctx->num_sms, ctx->stream));
            CD_CUDA(ozaki_slice_t(Y + (i0 - lo) * M * N, N, M * N, B, ctx->stream));
            CD_CUDA(ozaki_gemm(A, false, B, false, ctx->oz_p.as<double>(), N, v * N, 1.0, 0.0, err, ctx->num_sms,
                               ctx->stream));
            ctx->launches += 5;
            CD_RC(sum_batches(ctx, ctx->oz_p.as<double>(), (int)nb, v * N, scale, i0 > lo, dC + o * N));
        }
    }
    // W[i][Q][nu] into the Y buffer: A = Gamma_i^T (rows Q, K = a, strided by Mp),
    // B = C_vir^T (rows nu, K = a, strided by N), shared
    {
        OzakiOperand B = ozaki_operand(N, v, BN, 1);
        const size_t pa = operand_bytes(padded_rows(M, BM), padded_k(v));
        const int64_t ib = std::max<int64_t>(1, std::min<int64_t>(ni, (int64_t)(kSliceBytes / pa)));
        CD_ALLOC(ctx->oz_a, pa * ib, false);
        CD_ALLOC(ctx->oz_ea, sizeof(int) * (size_t)(padded_rows(M, BM) * ib), false);
        CD_ALLOC(ctx->oz_b, operand_bytes(B.Rp, B.Kp), false);
        CD_ALLOC(ctx->oz_eb, sizeof(int) * (size_t)B.Rp, false);
        B.q = ctx->oz_b.as<int8_t>();  B.e = ctx->oz_eb.as<int>();
        CD_CUDA(ozaki_slice_t(C + o * N, N, 0, B, ctx->stream));
        ctx->launches += 3;
        for (int64_t i0 = lo; i0 < hi; i0 += ib) {
            const int64_t nb = std::min(ib, hi - i0);
            OzakiOperand A = ozaki_operand(M, v, BM, (int)nb);
            A.q = ctx->oz_a.as<int8_t>();  A.e = ctx->oz_ea.as<int>();
            CD_CUDA(ozaki_slice_t(Gm + i0 * vp * Mp, Mp, vp * Mp, A, ctx->stream));
            CD_CUDA(ozaki_gemm(A, false, B, true, Y + (i0 - lo) * M * N, N, M * N, 1.0, 0.0, err, ctx->num_sms,
                               ctx->stream));
            ctx->launches += 4;
        }
        ctx->Y_spin = -1;
    }
    // dC[mu, i]: A = W_Q (rows i, K = nu), B = L_Q (rows mu, K = nu, strided by N)
    {
        const size_t pa = operand_bytes(padded_rows(ni, BM), padded_k(N));
        const size_t pb = operand_bytes(padded_rows(N, BN), padded_k(N));
        const size_t pp = sizeof(double) * (size_t)(ni * N);
        const int64_t nq_max = std::max<int64_t>(1, (int64_t)(2 * kSliceBytes / (pa + pb + pp)));
        const int64_t qc = vectors_chunk_size(ctx);
        // (batches are the z dimension of the transposed-slicing grid)
        const int64_t nq = std::min<int64_t>(std::min(nq_max, qc), 65535);
        CD_ALLOC(ctx->oz_a, pa * nq, false);
        CD_ALLOC(ctx->oz_b, pb * nq, false);
        CD_ALLOC(ctx->oz_p, pp * nq, false);
        CD_ALLOC(ctx->oz_ea, sizeof(int) * (size_t)(padded_rows(ni, BM) * nq), false);
        CD_ALLOC(ctx->oz_eb, sizeof(int) * (size_t)(padded_rows(N, BN) * nq), false);
        for (int64_t Q0 = 0; Q0 < M; Q0 += qc) {
            const int64_t mc = std::min(qc, M - Q0);
            const double* Lc = nullptr;
            CD_RC(vectors_chunk(ctx, Q0, mc, &Lc));
            for (int64_t q0 = 0; q0 < mc; q0 += nq) {
                const int64_t nb = std::min(nq, mc - q0);
                OzakiOperand A = ozaki_operand(ni, N, BM, (int)nb), B = ozaki_operand(N, N, BN, (int)nb);
                A.q = ctx->oz_a.as<int8_t>();  A.e = ctx->oz_ea.as<int>();
                B.q = ctx->oz_b.as<int8_t>();  B.e = ctx->oz_eb.as<int>();
                CD_CUDA(ozaki_slice(Y + (Q0 + q0) * N, M * N, N, A, ctx->num_sms, ctx->stream));
                CD_CUDA(ozaki_slice_t(Lc + q0 * N * N, N, N * N, B, ctx->stream));
                CD_CUDA(ozaki_gemm(A, false, B, false, ctx->oz_p.as<double>(), N, ni * N, 1.0, 0.0, err,
                                   ctx->num_sms, ctx->stream));
                ctx->launches += 5;
                CD_RC(sum_batches(ctx, ctx->oz_p.as<double>(), (int)nb, ni * N, scale, Q0 + q0 > 0, dC + lo * N));
            }
        }
    }
    int herr = 0;
    CD_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    if (herr)
        return set_error(MSHQC_CD_ERR_TIMEOUT, "int8 tensor-core transposed transform gave up waiting (site " +
                                                   std::to_string(herr) + ")");
    return MSHQC_CD_OK;
}

// dE/dC of one spin: the int8-slice transposed transforms for the mixed path
// (unless switched off), FP64 otherwise
int transposed_dispatch(mshqc_cd_ctx* ctx, int spin, double scale, double* dC, int precision) {
    if (precision == MSHQC_CD_FP16X3 && int8_transform_enabled(ctx))
        return transposed_transforms_i8(ctx, spin, scale, dC);
    return transposed_transforms(ctx, spin, scale, dC);
}

// ---------------------------------------------------------------------------
// backward building blocks (tensor-core and FP64 unrestricted passes)
// ---------------------------------------------------------------------------
struct BwdDims {
    int64_t o, v, vp;       // occupied, virtual, FP64 padding (64)
    int64_t VR, nby, VS;    // tensor-core staging: rows per i (128), column ranges (256) per j
};

BwdDims bwd_dims(const mshqc_cd_ctx* ctx, int spin) {
    BwdDims d;
    d.o = ctx->spin[spin].nocc;
    d.v = ctx->N - d.o;
    d.vp = ctx->spin[spin].vp;
    d.VR = cdiv(d.v, 128) * 128;
    d.nby = cdiv(d.VR, 256);
    d.VS = d.nby * 256;
    return d;
}

// BF16 hi/lo copy of one spin's MO vectors transposed to rows Q (RQ rows),
// K = (j, b) with b padded to VR: the B operand of the Gamma GEMM.
int make_bt(mshqc_cd_ctx* ctx, int spin, DevBuf& buf, int64_t RQ, const uint16_t** hi, const uint16_t** lo) {
    SpinState& s = ctx->spin[spin];
    const BwdDims d = bwd_dims(ctx, spin);
    const size_t nbt = (size_t)RQ * d.o * d.VR;
    CD_ALLOC(buf, 2 * nbt * sizeof(uint16_t), false);
    uint16_t* h = buf.as<uint16_t>();
    uint16_t* l = h + nbt;
    const int64_t threads = (d.o * d.VR / 16) * RQ * 2;
    const int blocks = (int)std::min<int64_t>(cdiv(threads, 256), (int64_t)ctx->num_sms * 16);
    begin_stage(ctx, ST_SPLIT);
    bt_split_kernel<<<blocks, 256, 0, ctx->stream>>>(s.B64.as<double>(), s.vp, ctx->Mp, (int)d.v, (int)ctx->M,
                                                     d.o, d.VR, RQ, h, l);
    end_stage(ctx);
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    *hi = h;
    *lo = l;
    return MSHQC_CD_OK;
}

// gamma[(i0 + R / VR, R % VR)][Q] (+)= sum_K A[R][K] BT[Q][K] for R < rows;
// a_rbs / b_rbs: K chunks per row block of A (128 rows) and of BT (256 rows),
// bhi / blo pointing at the first K chunk used
int launch_gamma(mshqc_cd_ctx* ctx, const uint16_t* ahi, const uint16_t* alo, int64_t a_rbs, const uint16_t* bhi,
                 const uint16_t* blo, int64_t b_rbs, int64_t RQ, int64_t K, int64_t rows, int64_t VR, int64_t v,
                 int64_t vp, int i0, double* gamma, int accumulate) {
    GammaTcArgs g{};
    g.Ahi = ahi;  g.Alo = alo;  g.Bhi = bhi;  g.Blo = blo;
    g.a_rbs = a_rbs;  g.b_rbs = b_rbs;
    g.nk = (int)(K / 16);
    g.KP = 32;
    g.nrb = (int)(rows / 128);
    g.nqb = (int)(RQ / 256);
    g.VR = (int)VR;  g.v = (int)v;  g.vp = (int)vp;  g.Mp = (int)ctx->Mp;  g.i0 = i0;
    g.gamma = gamma;
    g.err = ctx->flag.as<int>() + 2;
    g.accumulate = accumulate;
    const size_t gsm = gamma_tc::SMEM_BYTES;
    CD_CUDA(cudaFuncSetAttribute(gamma_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm));
    const int grid = (int)std::min<int64_t>((int64_t)g.nrb * g.nqb, ctx->num_sms);
    g.group = 16;
    if (const char* env = std::getenv("MSHQC_CD_GAMMA_GROUP")) g.group = std::max(1, std::atoi(env));
    pace_params(&g.pace_every, &g.pace_slack, "MSHQC_CD_PACE", true);
    if (g.pace_every > 0) {
        CD_ALLOC(ctx->pace, sizeof(int) * (size_t)grid, true);
        g.pace = ctx->pace.as<int>();
    }
    begin_stage(ctx, ST_GAMMA);
    gamma_tc_kernel<<<grid, gamma_tc::THREADS, gsm, ctx->stream>>>(g);
    end_stage(ctx);
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    return MSHQC_CD_OK;
}

// dE/de of one backward pass from its per-pair sums (amp_elem.cuh)
int reduce_deps(mshqc_cd_ctx* ctx, const double* prow, const double* pcol, const double* pocc, int64_t ox,
                int64_t oy, int64_t rsx, int64_t ksy, int64_t vx, int64_t vy, double* deps_x, double* deps_y) {
    const int64_t npairs = ox * oy;
    deps_rows_kernel<<<(unsigned)cdiv(vx, 128), 128, 0, ctx->stream>>>(prow, npairs, (int)rsx, (int)vx,
                                                                       deps_x + ox);
    deps_rows_kernel<<<(unsigned)cdiv(vy, 128), 128, 0, ctx->stream>>>(pcol, npairs, (int)ksy, (int)vy,
                                                                       deps_y + oy);
    deps_occ_kernel<<<(unsigned)cdiv(std::max(ox, oy), 128), 128, 0, ctx->stream>>>(pocc, (int)ox, (int)oy,
                                                                                    deps_x, deps_y);
    CD_CUDA(cudaGetLastError());
    ctx->launches += 3;
    return MSHQC_CD_OK;
}

// One mixed-precision backward pass over block pairs (I, J): rows i in I of
// spin sx, columns j in J of spin sy.  Per block pair: (ia|jb) tiles on the
// tensor cores (exact fixed point, FP32 staging), the element-wise amplitude
// pass, Gamma_sx[I] += amplitudes x B_sy[J] and, when `mirror`, the transposed
// amplitudes update Gamma_sy[J] += amplitudes^T x B_sx[I].
//  * same spin / restricted: blocks of b orbitals, I <= J only.  The amplitude
//    of pair (j, i) is the transpose of that of (i, j) (t^{ji}_{ba} =
//    t^{ij}_{ab}), so off-diagonal pairs are computed once and count twice;
//    this halves the integral tiles and the element-wise pass.
//  * opposite spin: row blocks I against all beta columns (no symmetry).
// Energies go to `partial` (ox * oy, one per ordered pair, zero where a
// mirrored pair stands in), dE/de to deps_x / deps_y.
template <int MODE>
int tc_backward_pass(mshqc_cd_ctx* ctx, int sx, int sy, const uint16_t* const btx[2],
                     const uint16_t* const bty[2], int64_t RQ, double* deps_x, double* deps_y,
                     double* partial) {
    constexpr bool kSym = MODE != AMP_OPPOSITE_SPIN;
    SpinState& X = ctx->spin[sx];
    SpinState& Y = ctx->spin[sy];
    const BwdDims dx = bwd_dims(ctx, sx), dy = bwd_dims(ctx, sy);
    const int64_t Mp = ctx->Mp;
    size_t free_b = 0, total_b = 0;
    CD_CUDA(cudaMemGetInfo(&free_b, &total_b));
    // the staging this pass reuses counts as available, so that the block size
    // of a repeated call does not shrink because the previous call holds it
    const size_t held = ctx->amp.bytes + ctx->amp2.bytes + ctx->ampT.bytes + ctx->ampT2.bytes + ctx->W.bytes;
    const size_t budget = std::min<size_t>((free_b + held) / 3, size_t(40) << 30);
    // block sizes: rows bI, columns bJ (all of them for the opposite spin)
    int64_t bI, bJ;
    tc_block_sizes(ctx, dx.o, dy.o, dx.VR, dy.VR, dy.VS, kSym, budget, &bI, &bJ);
    const size_t n_amp = sizeof(uint16_t) * (size_t)(bI * dx.VR) * (size_t)(bJ * dy.VR);
    CD_ALLOC(ctx->amp, n_amp, false);
    CD_ALLOC(ctx->amp2, n_amp, false);
    CD_ALLOC(ctx->ampT, n_amp, false);
    CD_ALLOC(ctx->ampT2, n_amp, false);
    CD_ALLOC(ctx->W, sizeof(float) * (size_t)(bI * dx.VR) * (size_t)(bJ * dy.VS), false);
    const int64_t npairs = dx.o * dy.o;
    CD_ALLOC(ctx->dsum, sizeof(double) * (size_t)(npairs * (dx.VR + dy.VR + 1)), true);
    CD_CUDA(cudaMemsetAsync(partial, 0, sizeof(double) * (size_t)npairs, ctx->stream));
    double* prow = ctx->dsum.as<double>();
    double* pcol = prow + npairs * dx.VR;
    double* pocc = pcol + npairs * dy.VR;
    if (X.B16_layout != 0 || Y.B16_layout != 0)
        return set_error(MSHQC_CD_ERR_STATE, "fixed-point operands not in the integral-tile layout");
    const size_t vsm = vtile_tc::SMEM_BYTES;
    CD_CUDA(cudaFuncSetAttribute(vtile_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsm));
    for (int64_t I0 = 0; I0 < dx.o; I0 += bI) {
        const int nI = (int)std::min<int64_t>(bI, dx.o - I0);
        for (int64_t J0 = kSym ? I0 : 0; J0 < dy.o; J0 += bJ) {
            if (!owns_next(ctx)) continue;
            const int nJ = (int)std::min<int64_t>(bJ, dy.o - J0);
            const bool mirror = !kSym || J0 != I0;
            // a diagonal block pair computes its pairs i <= j only; the
            // element-wise pass writes the (j, i) amplitudes as transposes
            const bool tri = kSym && J0 == I0;
            const int npl = tri ? nI * (nI + 1) / 2 : nI * nJ;
            VtileArgs a{};
            a.Xhi = X.Bhi.as<uint16_t>();  a.Xlo = X.Blo.as<uint16_t>();
            a.Yhi = Y.Bhi.as<uint16_t>();  a.Ylo = Y.Blo.as<uint16_t>();
            a.ex = X.expo.as<int>();  a.ey = Y.expo.as<int>();
            a.diag = sx == sy ? X.diag.as<double>() : nullptr;
            a.rows_x = (int)X.vp16;  a.rows_y = (int)Y.vp16;
            a.nqc = (int)(Mp / 16);
            a.j0 = (int)J0;  a.nbj = nJ;
            a.vx = (int)dx.v;  a.vy = (int)dy.v;
            a.VR = (int)dx.VR;  a.i0 = (int)I0;  a.nbi = nI;
            a.nbx = (int)(dx.VR / 128);  a.nby = (int)dy.nby;  a.VS = (int)dy.VS;
            a.S = ctx->W.as<float>();
            a.err = ctx->flag.as<int>();
            a.tri = tri ? 1 : 0;
            const int64_t vunits = (int64_t)npl * a.nbx * a.nby;
            const int vgrid = (int)std::min<int64_t>(vunits, ctx->num_sms);
            pace_params(&a.pace_every, &a.pace_slack, "MSHQC_CD_PACE_TILES", false);
            if (a.pace_every > 0) {
                CD_ALLOC(ctx->pace, sizeof(int) * (size_t)vgrid, true);
                a.pace = ctx->pace.as<int>();
            }
            begin_stage(ctx, ST_AMPLITUDE);
            vtile_tc_kernel<<<vgrid, vtile_tc::THREADS, vsm, ctx->stream>>>(a);
            end_stage(ctx);
            CD_CUDA(cudaGetLastError());
            ctx->launches++;
            AmpElemArgs e{};
            e.S = ctx->W.as<float>();
            e.ldS = (long long)nJ * dy.VS;
            e.rsx = (int)dx.VR;  e.csy = (int)dy.VS;  e.ksy = (int)dy.VR;
            e.ox = (int)dx.o;  e.oy = (int)dy.o;  e.vx = (int)dx.v;  e.vy = (int)dy.v;
            e.i0 = (int)I0;  e.nbi = nI;  e.j0 = (int)J0;  e.nbj = nJ;
            e.wgt = (kSym && mirror) ? 2.0 : 1.0;
            e.eox = X.eps.as<double>();  e.evx = e.eox + dx.o;
            e.eoy = Y.eps.as<double>();  e.evy = e.eoy + dy.o;
            e.Ahi = ctx->amp.as<uint16_t>();  e.Alo = ctx->amp2.as<uint16_t>();
            e.nkA = (long long)nJ * dy.VR / 16;
            if (mirror) {
                e.Thi = ctx->ampT.as<uint16_t>();  e.Tlo = ctx->ampT2.as<uint16_t>();
                e.nkT = (long long)nI * dx.VR / 16;
            } else if (tri) {
                e.Thi = e.Ahi;  e.Tlo = e.Alo;  e.nkT = e.nkA;
                e.tri = 1;
            }
            e.partial = partial;
            e.prow = prow;  e.pcol = pcol;  e.pocc = pocc;
            // split each pair's row tiles over several CTAs when the block
            // pair alone does not fill the GPU several times over
            const int ta = (int)(dx.VR / 32);
            int nch = 1;
            while (nch < 16 && 2 * nch <= ta && (int64_t)npl * nch < 8LL * ctx->num_sms) nch *= 2;
            e.nchunk = nch;
            if (nch > 1) {
                const size_t per = (size_t)npl * nch;
                CD_ALLOC(ctx->amp_chunks, sizeof(double) * per * ((size_t)dy.VR + 2), false);
                e.cpcol = ctx->amp_chunks.as<double>();
                e.cpart = e.cpcol + per * dy.VR;
                e.cpocc = e.cpart + per;
            }
            begin_stage(ctx, ST_AMP_ELEM);
            amp_elem_kernel<MODE, true><<<(unsigned)(npl * nch), 256, 0, ctx->stream>>>(e);
            CD_CUDA(cudaGetLastError());
            ctx->launches++;
            if (nch > 1) {
                amp_chunks_combine_kernel<<<(unsigned)cdiv((int64_t)npl * dy.VR, 256), 256, 0, ctx->stream>>>(e, npl);
                CD_CUDA(cudaGetLastError());
                ctx->launches++;
            }
            end_stage(ctx);
            // Gamma_sx[I] += A x B_sy[J]  (K range of J inside the transposed B of spin sy)
            // first K chunk of block J (I) inside a 256-row block of BT
            const size_t kJ = (size_t)J0 * dy.VR / 16 * 4096, kI = (size_t)I0 * dx.VR / 16 * 4096;
            const int64_t nkBy = dy.o * dy.VR / 16, nkBx = dx.o * dx.VR / 16;
            CD_RC(launch_gamma(ctx, e.Ahi, e.Alo, e.nkA, bty[0] + kJ, bty[1] + kJ, nkBy, RQ, (int64_t)nJ * dy.VR,
                               (int64_t)nI * dx.VR, dx.VR, dx.v, dx.vp, (int)I0, ctx->gam[sx].as<double>(), 1));
            if (mirror) {
                // Gamma_sy[J] += A^T x B_sx[I]
                CD_RC(launch_gamma(ctx, e.Thi, e.Tlo, e.nkT, btx[0] + kI, btx[1] + kI, nkBx, RQ,
                                   (int64_t)nI * dx.VR, (int64_t)nJ * dy.VR, dy.VR, dy.v, dy.vp, (int)J0,
                                   ctx->gam[sy].as<double>(), 1));
            }
        }
    }
    CD_RC(reduce_deps(ctx, prow, pcol, pocc, dx.o, dy.o, dx.VR, dy.VR, dx.v, dy.v, deps_x, deps_y));
    return MSHQC_CD_OK;
}

// The FP64 counterpart of tc_backward_pass, over the same block pairs: S =
// B_x[I] B_y[J]^T and the Gamma products as FP64 DMMA GEMMs around the
// element-wise pass.  A diagonal block pair of the symmetric modes forms S
// for j >= i only (one GEMM per row i), and the element-wise pass completes
// the amplitude block with the transposes.
template <int MODE>
int f64_backward_pass(mshqc_cd_ctx* ctx, int sx, int sy, double* deps_x, double* deps_y, double* partial) {
    constexpr bool kSym = MODE != AMP_OPPOSITE_SPIN;
    SpinState& X = ctx->spin[sx];
    SpinState& Y = ctx->spin[sy];
    const BwdDims dx = bwd_dims(ctx, sx), dy = bwd_dims(ctx, sy);
    const int64_t Mp = ctx->Mp;
    size_t free_b = 0, total_b = 0;
    CD_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t held = ctx->amp.bytes + ctx->W.bytes;
    const size_t budget = std::min<size_t>((free_b + held) / 3, size_t(40) << 30);
    int64_t bI, bJ;
    f64_block_sizes(ctx, dx.o, dy.o, dx.vp, dy.vp, kSym, budget, &bI, &bJ);
    const size_t n_stage = sizeof(double) * (size_t)(bI * dx.vp) * (size_t)(bJ * dy.vp);
    CD_ALLOC(ctx->W, n_stage, false);
    CD_ALLOC(ctx->amp, n_stage, false);
    const int64_t npairs = dx.o * dy.o;
    CD_ALLOC(ctx->dsum, sizeof(double) * (size_t)(npairs * (dx.vp + dy.vp + 1)), true);
    CD_CUDA(cudaMemsetAsync(partial, 0, sizeof(double) * (size_t)npairs, ctx->stream));
    double* prow = ctx->dsum.as<double>();
    double* pcol = prow + npairs * dx.vp;
    double* pocc = pcol + npairs * dy.vp;
    double* S = ctx->W.as<double>();
    double* A = ctx->amp.as<double>();
    for (int64_t I0 = 0; I0 < dx.o; I0 += bI) {
        const int nI = (int)std::min<int64_t>(bI, dx.o - I0);
        const double* XI = X.B64.as<double>() + I0 * dx.vp * Mp;
        for (int64_t J0 = kSym ? I0 : 0; J0 < dy.o; J0 += bJ) {
            if (!owns_next(ctx)) continue;
            const int nJ = (int)std::min<int64_t>(bJ, dy.o - J0);
            const bool mirror = !kSym || J0 != I0;
            const bool tri = kSym && J0 == I0;
            const int npl = tri ? nI * (nI + 1) / 2 : nI * nJ;
            const int64_t ldS = (int64_t)nJ * dy.vp;
            const double* YJ = Y.B64.as<double>() + J0 * dy.vp * Mp;
            // S[(i,a)][(j,b)] = sum_Q X[(i,a)][Q] Y[(j,b)][Q]
            begin_stage(ctx, ST_AMPLITUDE);
            for (int r = 0; r < (tri ? nI : 1); ++r) {
                GemmF64Args g{};
                g.M = (int)((tri ? 1 : nI) * dx.vp);  g.N = (int)((nJ - r) * dy.vp);  g.K = (int)Mp;  g.batch = 1;
                g.A = XI + (int64_t)r * dx.vp * Mp;  g.lda = Mp;  g.sA = 0;
                g.B = YJ + (int64_t)r * dy.vp * Mp;  g.ldb = Mp;  g.sB = 0;
                g.C = S + (int64_t)r * dx.vp * ldS + (int64_t)r * dy.vp;  g.ldc = ldS;  g.sC = 0;
                g.alpha = 1.0;  g.beta = 0.0;
                CD_CUDA(gemm_f64(g, true, true, ctx->stream));
                ctx->launches++;
            }
            end_stage(ctx);
            AmpElemArgs e{};
            e.S = S;
            e.ldS = ldS;
            e.rsx = (int)dx.vp;  e.csy = (int)dy.vp;  e.ksy = (int)dy.vp;
            e.ox = (int)dx.o;  e.oy = (int)dy.o;  e.vx = (int)dx.v;  e.vy = (int)dy.v;
            e.i0 = (int)I0;  e.nbi = nI;  e.j0 = (int)J0;  e.nbj = nJ;
            e.wgt = (kSym && mirror) ? 2.0 : 1.0;
            e.tri = tri ? 1 : 0;
            e.eox = X.eps.as<double>();  e.evx = e.eox + dx.o;
            e.eoy = Y.eps.as<double>();  e.evy = e.eoy + dy.o;
            e.A64 = A;  e.ldA = ldS;
            e.partial = partial;
            e.prow = prow;  e.pcol = pcol;  e.pocc = pocc;
            const int ta = (int)(dx.vp / 32);
            int nch = 1;
            while (nch < 16 && 2 * nch <= ta && (int64_t)npl * nch < 8LL * ctx->num_sms) nch *= 2;
            e.nchunk = nch;
            if (nch > 1) {
                const size_t per = (size_t)npl * nch;
                CD_ALLOC(ctx->amp_chunks, sizeof(double) * per * ((size_t)dy.vp + 2), false);
                e.cpcol = ctx->amp_chunks.as<double>();
                e.cpart = e.cpcol + per * dy.vp;
                e.cpocc = e.cpart + per;
            }
            begin_stage(ctx, ST_AMP_ELEM);
            amp_elem_kernel<MODE, false><<<(unsigned)(npl * nch), 256, 0, ctx->stream>>>(e);
            CD_CUDA(cudaGetLastError());
            ctx->launches++;
            if (nch > 1) {
                amp_chunks_combine_kernel<<<(unsigned)cdiv((int64_t)npl * dy.vp, 256), 256, 0, ctx->stream>>>(e, npl);
                CD_CUDA(cudaGetLastError());
                ctx->launches++;
            }
            end_stage(ctx);
            begin_stage(ctx, ST_GAMMA);
            // Gamma_x[(i,a)][Q] += sum_{(j,b) in J} t[(i,a)][(j,b)] Y[(j,b)][Q]
            GemmF64Args h{};
            h.M = (int)(nI * dx.vp);  h.N = (int)Mp;  h.K = (int)ldS;  h.batch = 1;
            h.A = A;  h.lda = ldS;  h.sA = 0;
            h.B = YJ;  h.ldb = Mp;  h.sB = 0;
            h.C = ctx->gam[sx].as<double>() + I0 * dx.vp * Mp;  h.ldc = Mp;  h.sC = 0;
            h.alpha = 1.0;  h.beta = 1.0;
            CD_CUDA(gemm_f64(h, true, false, ctx->stream));
            ctx->launches++;
            if (mirror) {
                // Gamma_y[(j,b)][Q] += sum_{(i,a) in I} t[(i,a)][(j,b)] X[(i,a)][Q]
                GemmF64Args k{};
                k.M = (int)ldS;  k.N = (int)Mp;  k.K = (int)(nI * dx.vp);  k.batch = 1;
                k.A = A;  k.lda = ldS;  k.sA = 0;
                k.B = XI;  k.ldb = Mp;  k.sB = 0;
                k.C = ctx->gam[sy].as<double>() + J0 * dy.vp * Mp;  k.ldc = Mp;  k.sC = 0;
                k.alpha = 1.0;  k.beta = 1.0;
                CD_CUDA(gemm_f64(k, false, false, ctx->stream));
                ctx->launches++;
            }
            end_stage(ctx);
        }
    }
    CD_RC(reduce_deps(ctx, prow, pcol, pocc, dx.o, dy.o, dx.vp, dy.vp, dx.v, dy.v, deps_x, deps_y));
    return MSHQC_CD_OK;
}

// Restricted FP64 gradient: one FP64 block-pair pass, then the transposed
// half transforms with dE/dB = 4 Gamma.
int gradient_restricted_f64(mshqc_cd_ctx* ctx, double* dC, double* deps, double* energy) {
    SpinState& s = ctx->spin[0];
    const int64_t N = ctx->N, Mp = ctx->Mp, o = s.nocc;
    CD_ALLOC(ctx->gam[0], sizeof(double) * (size_t)b_rows(ctx, o) * s.vp * Mp, true);
    CD_CUDA(cudaMemsetAsync(deps, 0, sizeof(double) * N, ctx->stream));
    CD_ALLOC(ctx->totals, sizeof(double) * 8, false);
    CD_ALLOC(ctx->partial, sizeof(double) * (size_t)(o * o), false);
    CD_RC(f64_backward_pass<AMP_RESTRICTED>(ctx, 0, 0, deps, deps, ctx->partial.as<double>()));
    reduce_total_kernel<<<1, 256, 0, ctx->stream>>>(ctx->partial.as<double>(), (int)(o * o), ctx->totals.as<double>());
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    CD_CUDA(cudaMemcpyAsync(energy, ctx->totals.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    begin_stage(ctx, ST_TRANSPOSED);
    CD_RC(transposed_dispatch(ctx, 0, 4.0, dC, MSHQC_CD_FP64));
    end_stage(ctx);
    return MSHQC_CD_OK;
}

// Restricted mixed-precision gradient: one tensor-core pass, then the FP64
// transposed transforms with dE/dB = 4 Gamma.
int gradient_restricted_tc(mshqc_cd_ctx* ctx, double* dC, double* deps, double* energy) {
    SpinState& s = ctx->spin[0];
    const BwdDims d = bwd_dims(ctx, 0);
    const int64_t N = ctx->N, Mp = ctx->Mp, RQ = round_up(ctx->M, 256);
    const uint16_t* bt[2] = {nullptr, nullptr};
    CD_RC(make_bt(ctx, 0, ctx->BT, RQ, &bt[0], &bt[1]));
    CD_ALLOC(ctx->gam[0], sizeof(double) * (size_t)b_rows(ctx, d.o) * s.vp * Mp, true);
    CD_CUDA(cudaMemsetAsync(deps, 0, sizeof(double) * N, ctx->stream));
    CD_ALLOC(ctx->flag, sizeof(int) * 4, true);
    CD_ALLOC(ctx->totals, sizeof(double) * 8, false);
    const int64_t tiles = d.o * d.o;   // one energy per pair (i, j)
    CD_ALLOC(ctx->partial, sizeof(double) * (size_t)tiles, false);
    CD_RC(tc_backward_pass<AMP_RESTRICTED>(ctx, 0, 0, bt, bt, RQ, deps, deps, ctx->partial.as<double>()));
    reduce_total_kernel<<<1, 256, 0, ctx->stream>>>(ctx->partial.as<double>(), (int)tiles, ctx->totals.as<double>());
    CD_CUDA(cudaGetLastError());
    ctx->launches++;
    int herr[4] = {0, 0, 0, 0};
    CD_CUDA(cudaMemcpyAsync(herr, ctx->flag.p, sizeof(herr), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaMemcpyAsync(energy, ctx->totals.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    if (herr[0] || herr[2])
        return set_error(MSHQC_CD_ERR_TIMEOUT, "tensor-core backward gave up waiting (site " +
                                                   std::to_string(herr[0] ? herr[0] : herr[2]) + ")");
    if (herr[1]) ctx->fixed_point_exact = 0;
    begin_stage(ctx, ST_TRANSPOSED);
    CD_RC(transposed_dispatch(ctx, 0, 4.0, dC, MSHQC_CD_FP16X3));
    end_stage(ctx);
    return MSHQC_CD_OK;
}

// Unrestricted gradient (CD-UMP2 energy, the OMP2 step): same-spin passes for
// alpha and beta and one opposite-spin pass, Gamma accumulated per spin, then
// the transposed transforms of each spin with dE/dB = 2 Gamma.  e3 receives
// ss_aa, ss_bb, os.
int gradient_unrestricted(mshqc_cd_ctx* ctx, int precision, double* const dC[2], double* const deps[2],
                          double* e3) {
    const BwdDims da = bwd_dims(ctx, 0), db = bwd_dims(ctx, 1);
    const int64_t N = ctx->N, Mp = ctx->Mp, RQ = round_up(ctx->M, 256);
    const bool tc = precision == MSHQC_CD_FP16X3;
    const uint16_t* bta[2] = {nullptr, nullptr};
    const uint16_t* btb[2] = {nullptr, nullptr};
    if (tc) {
        CD_RC(make_bt(ctx, 0, ctx->BT, RQ, &bta[0], &bta[1]));
        CD_RC(make_bt(ctx, 1, ctx->BT_b, RQ, &btb[0], &btb[1]));
    }
    CD_ALLOC(ctx->gam[0], sizeof(double) * (size_t)b_rows(ctx, da.o) * da.vp * Mp, true);
    CD_ALLOC(ctx->gam[1], sizeof(double) * (size_t)b_rows(ctx, db.o) * db.vp * Mp, true);
    for (int s = 0; s < 2; ++s) CD_CUDA(cudaMemsetAsync(deps[s], 0, sizeof(double) * N, ctx->stream));
    CD_ALLOC(ctx->flag, sizeof(int) * 4, true);
    CD_ALLOC(ctx->totals, sizeof(double) * 8, false);
    const int64_t n0 = da.o * da.o, n1 = db.o * db.o, n2 = da.o * db.o;   // one energy per pair
    CD_ALLOC(ctx->partial, sizeof(double) * (size_t)(n0 + n1 + n2), false);
    double* part = ctx->partial.as<double>();
    if (tc) {
        CD_RC(tc_backward_pass<AMP_SAME_SPIN>(ctx, 0, 0, bta, bta, RQ, deps[0], deps[0], part));
        CD_RC(tc_backward_pass<AMP_SAME_SPIN>(ctx, 1, 1, btb, btb, RQ, deps[1], deps[1], part + n0));
        CD_RC(tc_backward_pass<AMP_OPPOSITE_SPIN>(ctx, 0, 1, bta, btb, RQ, deps[0], deps[1], part + n0 + n1));
    } else {
        CD_RC(f64_backward_pass<AMP_SAME_SPIN>(ctx, 0, 0, deps[0], deps[0], part));
        CD_RC(f64_backward_pass<AMP_SAME_SPIN>(ctx, 1, 1, deps[1], deps[1], part + n0));
        CD_RC(f64_backward_pass<AMP_OPPOSITE_SPIN>(ctx, 0, 1, deps[0], deps[1], part + n0 + n1));
    }
    const int64_t offs[3] = {0, n0, n0 + n1}, cnt[3] = {n0, n1, n2};
    for (int k = 0; k < 3; ++k) {
        reduce_total_kernel<<<1, 256, 0, ctx->stream>>>(part + offs[k], (int)cnt[k], ctx->totals.as<double>() + k);
        CD_CUDA(cudaGetLastError());
        ctx->launches++;
    }
    int herr[4] = {0, 0, 0, 0};
    CD_CUDA(cudaMemcpyAsync(herr, ctx->flag.p, sizeof(herr), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaMemcpyAsync(e3, ctx->totals.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    if (herr[0] || herr[2])
        return set_error(MSHQC_CD_ERR_TIMEOUT, "tensor-core backward gave up waiting (site " +
                                                   std::to_string(herr[0] ? herr[0] : herr[2]) + ")");
    if (herr[1]) ctx->fixed_point_exact = 0;
    begin_stage(ctx, ST_TRANSPOSED);
    CD_RC(transposed_dispatch(ctx, 0, 2.0, dC[0], precision));
    CD_RC(transposed_dispatch(ctx, 1, 2.0, dC[1], precision));
    end_stage(ctx);
    return MSHQC_CD_OK;
}

// The shares of a partitioned gradient call.  Enumerates the backward's units
// in the order the passes visit them, with the partitioned block sizes (a
// function of the dimensions and the rank count only), weighs each by its
// tensor-core or DMMA work (integral tiles + Gamma products, in (i, j) pair
// units: a diagonal block pair has no mirrored Gamma product), and deals them
// out longest first to the least-loaded rank (ties to the lower rank).  Every
// rank computes the same plan and keeps its own units.
int plan_partition(mshqc_cd_ctx* ctx, int kind, int precision) {
    std::vector<double> cost;
    const bool unres = kind == MSHQC_CD_UNRESTRICTED;
    auto tc_pass = [&](int sx, int sy, bool sym) {
        const BwdDims dx = bwd_dims(ctx, sx), dy = bwd_dims(ctx, sy);
        int64_t bI, bJ;
        tc_block_sizes(ctx, dx.o, dy.o, dx.VR, dy.VR, dy.VS, sym, 0, &bI, &bJ);
        for (int64_t I0 = 0; I0 < dx.o; I0 += bI) {
            const int64_t nI = std::min(bI, dx.o - I0);
            for (int64_t J0 = sym ? I0 : 0; J0 < dy.o; J0 += bJ) {
                const int64_t nJ = std::min(bJ, dy.o - J0);
                // integral tiles of the pairs computed + Gamma products
                if (sym && J0 == I0)
                    cost.push_back(0.5 * (double)nI * (nI + 1) + (double)nI * nI);
                else
                    cost.push_back(3.0 * nI * nJ);
            }
        }
    };
    // the FP64 passes visit the same kind of units; per block pair: S GEMM
    // (half of it on a diagonal block pair) + Gamma products
    auto f64_pass = [&](int sx, int sy, bool sym) {
        const BwdDims dx = bwd_dims(ctx, sx), dy = bwd_dims(ctx, sy);
        int64_t bI, bJ;
        f64_block_sizes(ctx, dx.o, dy.o, dx.vp, dy.vp, sym, 0, &bI, &bJ);
        for (int64_t I0 = 0; I0 < dx.o; I0 += bI) {
            const int64_t nI = std::min(bI, dx.o - I0);
            for (int64_t J0 = sym ? I0 : 0; J0 < dy.o; J0 += bJ) {
                const int64_t nJ = std::min(bJ, dy.o - J0);
                if (sym && J0 == I0)
                    cost.push_back(0.5 * (double)nI * (nI + 1) + (double)nI * nI);
                else
                    cost.push_back(3.0 * nI * nJ);
            }
        }
    };
    if (!unres && precision == MSHQC_CD_FP64) {
        f64_pass(0, 0, true);
    } else if (!unres) {
        tc_pass(0, 0, true);
    } else if (precision == MSHQC_CD_FP16X3) {
        tc_pass(0, 0, true);
        tc_pass(1, 1, true);
        tc_pass(0, 1, false);
    } else {
        f64_pass(0, 0, true);
        f64_pass(1, 1, true);
        f64_pass(0, 1, false);
    }
    std::vector<size_t> order(cost.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
    std::vector<double> load((size_t)ctx->part_size, 0.0);
    ctx->part_owned.assign(cost.size(), 0);
    for (size_t k : order) {
        const size_t r = (size_t)(std::min_element(load.begin(), load.end()) - load.begin());
        load[r] += cost[k];
        if ((int)r == ctx->part_rank) ctx->part_owned[k] = 1;
    }
    return MSHQC_CD_OK;
}

}  // namespace

int run_gradient(mshqc_cd_ctx* ctx, int kind, int precision, mshqc_cd_energy* e_out, double* dC_a,
                 double* dC_b, double* deps_a, double* deps_b, int where) {
    if (kind != MSHQC_CD_RESTRICTED && kind != MSHQC_CD_UNRESTRICTED)
        return set_error(MSHQC_CD_ERR_ARG, "unknown kind");
    const bool unres = kind == MSHQC_CD_UNRESTRICTED;
    CD_RC(require_inputs(ctx, 0));
    if (unres) CD_RC(require_inputs(ctx, 1));
    const int64_t N = ctx->N;
    // the partition applies to this call's backward only
    struct PartitionScope {
        mshqc_cd_ctx* c;
        explicit PartitionScope(mshqc_cd_ctx* x) : c(x) { c->part_active = c->part_size > 1; c->part_next = 0; }
        ~PartitionScope() { c->part_active = false; }
    } part_scope(ctx);
    cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[1], e2 = ctx->ev[2];
    reset_stages(ctx);
    CD_CUDA(cudaEventRecord(e0, ctx->stream));
    CD_RC(ensure_transform(ctx, 0, precision));
    if (unres) CD_RC(ensure_transform(ctx, 1, precision));
    CD_CUDA(cudaEventRecord(e1, ctx->stream));
    if (ctx->part_active) CD_RC(plan_partition(ctx, kind, precision));
    double* dC[2] = {nullptr, nullptr};
    double* de[2] = {nullptr, nullptr};
    for (int s = 0; s < (unres ? 2 : 1); ++s) {
        CD_ALLOC(ctx->grad[s], sizeof(double) * (size_t)(N * N + N), false);
        dC[s] = ctx->grad[s].as<double>();
        de[s] = dC[s] + N * N;
    }
    double e3[3] = {0.0, 0.0, 0.0};
    double energy = 0.0;
    ctx->fixed_point_exact = 1;
    if (unres) {
        CD_RC(gradient_unrestricted(ctx, precision, dC, de, e3));
        energy = e3[0] + e3[1] + e3[2];
    } else if (precision == MSHQC_CD_FP64) {
        CD_RC(gradient_restricted_f64(ctx, dC[0], de[0], &energy));
    } else {
        CD_RC(gradient_restricted_tc(ctx, dC[0], de[0], &energy));
    }
    if (ctx->part_active && ctx->part_next != (int64_t)ctx->part_owned.size())
        return set_error(MSHQC_CD_ERR_STATE, "partition plan covers " + std::to_string(ctx->part_owned.size()) +
                                                 " units, the backward visited " + std::to_string(ctx->part_next));
    CD_CUDA(cudaEventRecord(e2, ctx->stream));
    CD_CUDA(cudaEventSynchronize(e2));
    collect_stages(ctx);
    if (e_out) {
        std::memset(e_out, 0, sizeof(*e_out));
        e_out->total = energy;
        if (unres) {
            e_out->ss_aa = e3[0];
            e_out->ss_bb = e3[1];
            e_out->os = e3[2];
        }
        float t01 = 0, t12 = 0;
        CD_CUDA(cudaEventElapsedTime(&t01, e0, e1));
        CD_CUDA(cudaEventElapsedTime(&t12, e1, e2));
        e_out->ms_transform = t01;
        e_out->ms_energy = t12;
        e_out->ms_total = t01 + t12;
    }
    CD_RC(download(ctx, dC_a, dC[0], sizeof(double) * N * N, where));
    CD_RC(download(ctx, deps_a, de[0], sizeof(double) * N, where));
    if (unres) {
        CD_RC(download(ctx, dC_b, dC[1], sizeof(double) * N * N, where));
        CD_RC(download(ctx, deps_b, de[1], sizeof(double) * N, where));
    }
    return MSHQC_CD_OK;
}

}  // namespace mshqc_cd
