// Internal state of a libmshqc_cuda context (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/mshqc_cd.h"

namespace mshqc_cd {

// Grow-only device allocation: a context allocates on the first call at a
// given size and reuses the memory afterwards.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t nbytes, bool zero, cudaStream_t st);
    void release();
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct DeviceGuard {
    int prev = 0, target = 0;
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
};

struct SpinState {
    DevBuf C, eps;          // N*N column-major, N
    int64_t nocc = 0;
    bool set = false;
    // FP64 MO vectors [i][a][Q] (a padded to vp, Q to Mp)
    DevBuf B64;
    int64_t vp = 0;
    bool B64_valid = false;
    int B64_prec = 0;       // MSHQC_CD_FP64: FP64 products; MSHQC_CD_FP16X3: int8-slice products
    // fixed-point hi/lo (BF16 carriers) of the MO vectors for the tensor-core path
    DevBuf Bhi, Blo;        // Blo unused in the pair layout (hi and lo interleaved in Bhi)
    DevBuf expo;            // per-row power-of-two exponents [o][rows]
    DevBuf diag;            // exact (ia|ia) [o][rows]
    DevBuf norms;           // sum hi^2, sum lo^2 per row [2][o][rows]
    int64_t vp16 = 0, Mp16 = 0;
    double max_norm_hi = 0, max_norm_lo = 0;
    bool B16_valid = false;
    int B16_layout = 0;     // 0: integral-tile layout, 1: pair layout (split_bf16.cuh)
    void invalidate() {
        B64_valid = false;
        B16_valid = false;
    }
};

}  // namespace mshqc_cd

struct mshqc_cd_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6] = {};
    void* bounce[2] = {nullptr, nullptr};
    cudaEvent_t bounce_ev[2] = {nullptr, nullptr};

    int64_t N = 0, M = 0, Mp = 0;
    bool L_set = false;
    int64_t launches = 0;           // kernels launched by this context
    // per-stage device timing of the last call (see mshqc_cd_stage_times)
    double stage_ms[8] = {};
    int64_t stage_n[8] = {};        // timed intervals per stage of the last call
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, int>> ev_marks;   // (stage, index of the start event)
    size_t ev_used = 0;
    mshqc_cd::DevBuf L;             // [Q][N*N] FP64 (stored vectors)
    bool L_gen = false;             // vectors generated on the device, never stored
    uint64_t gen_seed = 0;
    mshqc_cd::DevBuf gen_scale;     // sigma * 10^(-6 Q / M) per Q (generated vectors)
    mshqc_cd::DevBuf Lchunk;        // one generated chunk of vectors
    mshqc_cd::SpinState spin[2];

    // workspaces
    mshqc_cd::DevBuf Y;             // half-transformed vectors
    int Y_spin = -1;                // spin whose Y is in the buffer (-1: none)
    mshqc_cd::DevBuf scratch;       // uploads / unpacking
    mshqc_cd::DevBuf tables;        // pair and block tables
    mshqc_cd::DevBuf partial;       // per-unit energies
    mshqc_cd::DevBuf pair_sum;      // per-pair energies
    mshqc_cd::DevBuf totals;        // scalar results
    mshqc_cd::DevBuf flag;          // error / NaN flags
    mshqc_cd::DevBuf pace;          // wave-pacing progress counters of the persistent tile kernels
    mshqc_cd::DevBuf amp;           // backward: staged amplitudes
    mshqc_cd::DevBuf gam[2];        // backward: Gamma per spin
    mshqc_cd::DevBuf BT;            // backward: transposed MO vectors (hi/lo BF16), alpha
    mshqc_cd::DevBuf BT_b;          // backward: the same for beta
    mshqc_cd::DevBuf amp2;          // backward: second half of the staging (lo)
    mshqc_cd::DevBuf ampT, ampT2;   // backward: transposed opposite-spin amplitudes (hi, lo)
    mshqc_cd::DevBuf dsum;          // backward: per-pair row / column / total sums for dE/de
    mshqc_cd::DevBuf amp_chunks;    // backward: per-chunk column sums, energies, totals of split pairs
    mshqc_cd::DevBuf W;             // backward: integral staging / C_vir-contracted Gamma
    mshqc_cd::DevBuf grad[4];       // backward: dC / deps per spin
    mshqc_cd::DevBuf diag_os;       // sum_Q B_alpha[i][a] B_beta[i][a] (opposite-spin diagonal)
    mshqc_cd::DevBuf Hcore;         // OMP2: core Hamiltonian N*N
    bool H_set = false;
    mshqc_cd::DevBuf opdm;          // OMP2: OPDM blocks, densities, Fock matrices
    mshqc_cd::DevBuf omp2_ws;       // OMP2: split-K partials, rotation work matrices
    mshqc_cd::DevBuf Zt;            // OMP2: P L^Q for every Q (M*N*N)
    mshqc_cd::DevBuf oz_a, oz_b;    // int8 slices of the transform operands (orbitals, vectors)
    mshqc_cd::DevBuf oz_ea, oz_eb;  // their row exponents
    mshqc_cd::DevBuf oz_flag;       // int8-slice product error flag
    mshqc_cd::DevBuf oz_p;          // per-batch FP64 partial products (transposed transforms)
    bool diag_os_valid = false;
    int fixed_point_exact = 1;      // Cauchy-Schwarz bound of the last tensor-core pass held
    // share of the backward computed by this context (mshqc_cd_set_partition):
    // the units (block pairs, or occupied blocks of the FP64 passes) of a
    // gradient call are numbered from 0 in the order the passes visit them;
    // part_owned[k] says whether unit k is this rank's (a cost-balanced plan
    // that every rank computes alike, see plan_partition in cd_mp2.cu)
    int part_rank = 0, part_size = 1;
    bool part_active = false;
    int64_t part_next = 0;
    std::vector<uint8_t> part_owned;
    // host collectives (mshqc_cd_set_collectives): with them the transforms
    // of a partitioned gradient are shared over occupied orbitals too
    mshqc_cd_collectives coll{};
    bool coll_set = false;
    int64_t Y_lo = 0, Y_hi = 0;     // occupied orbitals whose half-transformed vectors Y holds

    std::vector<double> pair_energy[3];  // host copies, row-major [i][j]

    void invalidate_all() {
        spin[0].invalidate();
        spin[1].invalidate();
        diag_os_valid = false;
        Y_spin = -1;
        for (auto& p : pair_energy) p.clear();
    }
    size_t held_bytes() const {
        size_t b = L.bytes + Y.bytes + scratch.bytes + tables.bytes + partial.bytes +
                   pair_sum.bytes + totals.bytes + flag.bytes + amp.bytes + amp2.bytes + BT.bytes + W.bytes;
        for (const auto& s : spin)
            b += s.C.bytes + s.eps.bytes + s.B64.bytes + s.Bhi.bytes + s.Blo.bytes + s.expo.bytes +
                 s.diag.bytes + s.norms.bytes;
        b += diag_os.bytes + oz_a.bytes + oz_b.bytes + oz_ea.bytes + oz_eb.bytes + oz_p.bytes;
        for (const auto& g : gam) b += g.bytes;
        for (const auto& g : grad) b += g.bytes;
        return b;
    }
    void release_all() {
        for (auto& e : ev_pool)
            if (e) cudaEventDestroy(e);
        ev_pool.clear();
        L.release();
        Y.release();
        scratch.release();
        tables.release();
        partial.release();
        pair_sum.release();
        totals.release();
        flag.release();
        pace.release();
        amp.release();
        BT.release();
        amp2.release();
        BT_b.release();
        ampT.release();
        ampT2.release();
        dsum.release();
        amp_chunks.release();
        W.release();
        for (auto& s : spin) {
            s.C.release();
            s.eps.release();
            s.B64.release();
            s.Bhi.release();
            s.Blo.release();
            s.expo.release();
            s.diag.release();
            s.norms.release();
        }
        diag_os.release();
        Hcore.release();
        gen_scale.release();
        Lchunk.release();
        opdm.release();
        omp2_ws.release();
        Zt.release();
        oz_a.release();
        oz_b.release();
        oz_ea.release();
        oz_eb.release();
        oz_flag.release();
        oz_p.release();
        for (auto& g : gam) g.release();
        for (auto& g : grad) g.release();
    }
};

namespace mshqc_cd {
enum Stage { ST_TRANSFORM = 0, ST_SPLIT, ST_PAIR, ST_AMPLITUDE, ST_GAMMA, ST_TRANSPOSED, ST_OTHER, ST_AMP_ELEM };
// stage timing: begin_stage/end_stage record events on the context stream;
// collect_stages (after a synchronize) folds them into ctx->stage_ms
void reset_stages(mshqc_cd_ctx* ctx);
void begin_stage(mshqc_cd_ctx* ctx, int stage);
void end_stage(mshqc_cd_ctx* ctx);
void collect_stages(mshqc_cd_ctx* ctx);
int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);
int upload(mshqc_cd_ctx* ctx, void* dst, const void* src, size_t nbytes);
int download(mshqc_cd_ctx* ctx, void* dst, const void* src, size_t nbytes, int where);
int check_finite_device(mshqc_cd_ctx* ctx, const double* x, int64_t n, const char* what);

// status helpers for functions returning an MSHQC_CD_* code (CD_ALLOC needs
// a `ctx` in scope)
#define CD_CUDA(call)                                                     \
    do {                                                                  \
        cudaError_t _e = (call);                                          \
        if (_e != cudaSuccess) return cuda_error(_e, #call);              \
    } while (0)
#define CD_ALLOC(buf, nbytes, zero)                                                        \
    do {                                                                                   \
        cudaError_t _e = (buf).reserve((nbytes), (zero), ctx->stream);                     \
        if (_e == cudaErrorMemoryAllocation)                                               \
            return set_error(MSHQC_CD_ERR_ALLOC, "device allocation of " +                 \
                                                     std::to_string((size_t)(nbytes)) +    \
                                                     " bytes failed");                     \
        if (_e != cudaSuccess) return cuda_error(_e, "workspace");                         \
    } while (0)
#define CD_RC(x)             \
    do {                     \
        int _rc = (x);       \
        if (_rc) return _rc; \
    } while (0)

// implemented in cd_mp2.cu
// layout: of the fixed-point operands of a mixed-precision request
// (0: integral tiles of the backward, 1: fused pair energies)
int ensure_transform(mshqc_cd_ctx* ctx, int spin, int precision, int layout = 0);
int run_energy(mshqc_cd_ctx* ctx, int kind, int precision, mshqc_cd_energy* out);
int run_gradient(mshqc_cd_ctx* ctx, int kind, int precision, mshqc_cd_energy* e_out,
                 double* dC_a, double* dC_b, double* deps_a, double* deps_b, int where);
int invalidate_spin(mshqc_cd_ctx* ctx, int spin);   // orbitals of `spin` changed on the device

// implemented in cd_vectors.cu: the vectors Q0 .. Q0 + mc - 1 (N*N doubles
// each, contiguous): the stored array, or a chunk generated into ctx->Lchunk
// (valid until the next call); vectors_chunk_size is the chunk to ask for.
int64_t vectors_chunk_size(const mshqc_cd_ctx* ctx);
int vectors_chunk(mshqc_cd_ctx* ctx, int64_t Q0, int64_t mc, const double** out);
}  // namespace mshqc_cd
