// C ABI of the B200 Cholesky-vector MP2 library (declared in include/mshqc_cd.h).
//
// Device data layout (HBM):
//   L      [Q][mu*N + nu] FP64, the reference CholeskyERI order; the transforms
//          read vector Q as the column-major map Lmap[mu,nu] = L[nu*N + mu] of
//          reference src/mp2/cholesky_rmp2.cc:85 (identical for symmetric L).
//   Y_s    [i][Q][nu]  = sum_mu C[mu,i] Lmap^Q[mu,nu]   (half-transformed, FP64)
//   B_s    [i][a][Q]   FP64, a padded to vp (multiple of 64) and Q to Mp
//          (multiple of 16) with zeros, so the pair kernels need no bounds
//          checks in their main loops.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mshqc_cd.h"
#include "cd_common.cuh"
#include "cd_internal.h"

using namespace mshqc_cd;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
namespace {
thread_local std::string g_last_error = "";
}

namespace mshqc_cd {
void reset_stages(mshqc_cd_ctx* ctx) {
    for (double& t : ctx->stage_ms) t = 0.0;
    for (int64_t& n : ctx->stage_n) n = 0;
    ctx->ev_marks.clear();
    ctx->ev_used = 0;
}
static cudaEvent_t next_event(mshqc_cd_ctx* ctx) {
    if (ctx->ev_used == ctx->ev_pool.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        ctx->ev_pool.push_back(e);
    }
    return ctx->ev_pool[ctx->ev_used++];
}
void begin_stage(mshqc_cd_ctx* ctx, int stage) {
    const size_t idx = ctx->ev_used;
    cudaEvent_t e = next_event(ctx);
    if (!e) return;
    cudaEventRecord(e, ctx->stream);
    ctx->ev_marks.push_back({stage, (int)idx});
}
void end_stage(mshqc_cd_ctx* ctx) {
    cudaEvent_t e = next_event(ctx);
    if (e) cudaEventRecord(e, ctx->stream);
}
void collect_stages(mshqc_cd_ctx* ctx) {
    for (const auto& m : ctx->ev_marks) {
        if ((size_t)m.second + 1 >= ctx->ev_used) continue;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, ctx->ev_pool[m.second], ctx->ev_pool[m.second + 1]) == cudaSuccess) {
            ctx->stage_ms[m.first] += ms;
            ctx->stage_n[m.first] += 1;
        }
    }
    ctx->ev_marks.clear();
    ctx->ev_used = 0;
}

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
int cuda_error(cudaError_t e, const char* what) {
    return set_error(MSHQC_CD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

cudaError_t DevBuf::reserve(size_t nbytes, bool zero, cudaStream_t st) {
    if (nbytes <= bytes) {
        if (zero && nbytes) return cudaMemsetAsync(p, 0, nbytes, st);
        return cudaSuccess;
    }
    release();
    cudaError_t e = cudaMalloc(&p, nbytes);
    if (e != cudaSuccess) {
        // the caller reports the failure; clear the runtime's last error so
        // that the next cudaGetLastError() after a kernel launch does not
        // return it again
        (void)cudaGetLastError();
        p = nullptr;
        bytes = 0;
        return e;
    }
    bytes = nbytes;
    if (zero) return cudaMemsetAsync(p, 0, nbytes, st);
    return cudaSuccess;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

DeviceGuard::DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
    target = dev;
}
DeviceGuard::~DeviceGuard() {
    if (prev != target) cudaSetDevice(prev);
}
}  // namespace mshqc_cd

#define CD_CHECK_CTX()                                                                  \
    do {                                                                                \
        if (!ctx) return set_error(MSHQC_CD_ERR_ARG, "null context");                   \
    } while (0)

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
namespace {

// packed upper triangle (mu <= nu, row by row) -> full symmetric N*N
__global__ void unpack_vectors_kernel(const double* __restrict__ packed, double* __restrict__ full,
                                      int64_t N, int64_t nq) {
    const int64_t tri = N * (N + 1) / 2;
    const int64_t total = nq * N * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = t / (N * N);
        const int64_t r = t % (N * N);
        int64_t mu = r / N, nu = r % N;
        if (mu > nu) {
            int64_t tmp = mu;
            mu = nu;
            nu = tmp;
        }
        const int64_t idx = mu * N - mu * (mu - 1) / 2 + (nu - mu);
        full[t] = packed[q * tri + idx];
    }
}

__global__ void count_nonfinite_kernel(const double* __restrict__ x, int64_t n,
                                       unsigned long long* __restrict__ bad) {
    unsigned long long local = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x)
        local += isfinite(x[t]) ? 0ull : 1ull;
    if (local) atomicAdd(bad, local);
}

bool host_all_finite(const double* x, int64_t n) {
    for (int64_t k = 0; k < n; ++k)
        if (!std::isfinite(x[k])) return false;
    return true;
}

bool is_device_pointer(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

bool is_pinned_host(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

}  // namespace

namespace mshqc_cd {
// Host -> device copy on the context stream.  Pinned sources go straight to
// the copy engine; pageable ones are staged through two pinned bounce buffers
// so the CPU memcpy of one chunk overlaps the DMA of the other.
int upload(mshqc_cd_ctx* ctx, void* dst, const void* src, size_t nbytes) {
    if (nbytes == 0) return MSHQC_CD_OK;
    if (is_pinned_host(src) || nbytes <= (size_t(4) << 20)) {
        CD_CUDA(cudaMemcpyAsync(dst, src, nbytes, cudaMemcpyHostToDevice, ctx->stream));
        CD_CUDA(cudaStreamSynchronize(ctx->stream));
        return MSHQC_CD_OK;
    }
    const size_t chunk = size_t(64) << 20;
    if (!ctx->bounce[0]) {
        for (int b = 0; b < 2; ++b) {
            CD_CUDA(cudaMallocHost(&ctx->bounce[b], chunk));
            CD_CUDA(cudaEventCreateWithFlags(&ctx->bounce_ev[b], cudaEventDisableTiming));
            CD_CUDA(cudaEventRecord(ctx->bounce_ev[b], ctx->stream));
        }
    }
    size_t off = 0;
    int b = 0;
    while (off < nbytes) {
        const size_t n = std::min(chunk, nbytes - off);
        CD_CUDA(cudaEventSynchronize(ctx->bounce_ev[b]));
        std::memcpy(ctx->bounce[b], static_cast<const char*>(src) + off, n);
        CD_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, ctx->bounce[b], n,
                                cudaMemcpyHostToDevice, ctx->stream));
        CD_CUDA(cudaEventRecord(ctx->bounce_ev[b], ctx->stream));
        off += n;
        b ^= 1;
    }
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}

int download(mshqc_cd_ctx* ctx, void* dst, const void* src, size_t nbytes, int where) {
    if (nbytes == 0 || !dst) return MSHQC_CD_OK;
    CD_CUDA(cudaMemcpyAsync(dst, src, nbytes,
                            where == MSHQC_CD_DEVICE ? cudaMemcpyDeviceToDevice
                                                     : cudaMemcpyDeviceToHost,
                            ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}

int check_finite_device(mshqc_cd_ctx* ctx, const double* x, int64_t n, const char* what) {
    CD_ALLOC(ctx->flag, sizeof(unsigned long long), true);
    auto* bad = static_cast<unsigned long long*>(ctx->flag.p);
    const int blocks = (int)std::min<int64_t>(4 * 148, std::max<int64_t>(1, cdiv(n, 256)));
    count_nonfinite_kernel<<<blocks, 256, 0, ctx->stream>>>(x, n, bad);
    ctx->launches++;
    CD_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    CD_CUDA(cudaMemcpyAsync(&h, bad, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h) return set_error(MSHQC_CD_ERR_NUMERIC, std::string(what) + " contains NaN/Inf");
    return MSHQC_CD_OK;
}
}  // namespace mshqc_cd

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
extern "C" {

const char* mshqc_cd_last_error(void) { return g_last_error.c_str(); }
int mshqc_cd_abi_version(void) { return MSHQC_CD_ABI_VERSION; }

int mshqc_cd_ctx_create(int device, mshqc_cd_ctx** out) {
    if (!out) return set_error(MSHQC_CD_ERR_ARG, "out is null");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(MSHQC_CD_ERR_UNSUPPORTED, "no CUDA device available");
    }
    if (device < 0 || device >= ndev)
        return set_error(MSHQC_CD_ERR_ARG, "device index out of range");
    cudaDeviceProp prop;
    CD_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10)
        return set_error(MSHQC_CD_ERR_UNSUPPORTED,
                         "libmshqc_cuda is built for sm_100a (B200); device is sm_" +
                             std::to_string(prop.major * 10 + prop.minor));
    DeviceGuard g(device);
    auto* ctx = new (std::nothrow) mshqc_cd_ctx();
    if (!ctx) return set_error(MSHQC_CD_ERR_ALLOC, "host allocation failed");
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_error(e, "cudaStreamCreate");
    }
    ctx->stream = ctx->own;
    for (auto& ev : ctx->ev) {
        e = cudaEventCreate(&ev);
        if (e != cudaSuccess) {
            delete ctx;
            return cuda_error(e, "cudaEventCreate");
        }
    }
    *out = ctx;
    return MSHQC_CD_OK;
}

int mshqc_cd_ctx_destroy(mshqc_cd_ctx* ctx) {
    if (!ctx) return MSHQC_CD_OK;
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->release_all();
    for (auto& ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    for (int b = 0; b < 2; ++b) {
        if (ctx->bounce[b]) cudaFreeHost(ctx->bounce[b]);
        if (ctx->bounce_ev[b]) cudaEventDestroy(ctx->bounce_ev[b]);
    }
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
    return MSHQC_CD_OK;
}

int mshqc_cd_set_stream(mshqc_cd_ctx* ctx, void* stream) {
    CD_CHECK_CTX();
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own;
    return MSHQC_CD_OK;
}

int mshqc_cd_set_partition(mshqc_cd_ctx* ctx, int rank, int nranks) {
    CD_CHECK_CTX();
    if (nranks < 1 || rank < 0 || rank >= nranks)
        return set_error(MSHQC_CD_ERR_ARG, "partition needs 0 <= rank < nranks");
    ctx->part_rank = rank;
    ctx->part_size = nranks;
    return MSHQC_CD_OK;
}

int mshqc_cd_set_collectives(mshqc_cd_ctx* ctx, const mshqc_cd_collectives* ops) {
    CD_CHECK_CTX();
    if (ops && (!ops->allgather || !ops->reduce_scatter))
        return set_error(MSHQC_CD_ERR_ARG, "collectives need allgather and reduce_scatter");
    ctx->coll_set = ops != nullptr;
    ctx->coll = ops ? *ops : mshqc_cd_collectives{};
    return MSHQC_CD_OK;
}

int mshqc_cd_stage_times(mshqc_cd_ctx* ctx, double* ms_out, int n_out) {
    CD_CHECK_CTX();
    if (!ms_out || n_out < 0) return set_error(MSHQC_CD_ERR_ARG, "bad output");
    for (int k = 0; k < n_out && k < 8; ++k) ms_out[k] = ctx->stage_ms[k];
    return MSHQC_CD_OK;
}

int mshqc_cd_stage_counts(mshqc_cd_ctx* ctx, int64_t* n_out, int n) {
    CD_CHECK_CTX();
    if (!n_out || n < 0) return set_error(MSHQC_CD_ERR_ARG, "bad output");
    for (int k = 0; k < n && k < 8; ++k) n_out[k] = ctx->stage_n[k];
    return MSHQC_CD_OK;
}

int mshqc_cd_mixed_exact(mshqc_cd_ctx* ctx, int* exact) {
    CD_CHECK_CTX();
    if (!exact) return set_error(MSHQC_CD_ERR_ARG, "exact is null");
    *exact = ctx->fixed_point_exact;
    return MSHQC_CD_OK;
}

int mshqc_cd_launch_count(mshqc_cd_ctx* ctx, int64_t* count) {
    CD_CHECK_CTX();
    if (!count) return set_error(MSHQC_CD_ERR_ARG, "count is null");
    *count = ctx->launches;
    return MSHQC_CD_OK;
}

int mshqc_cd_device_bytes(mshqc_cd_ctx* ctx, int64_t* bytes) {
    CD_CHECK_CTX();
    if (!bytes) return set_error(MSHQC_CD_ERR_ARG, "bytes is null");
    *bytes = (int64_t)ctx->held_bytes();
    return MSHQC_CD_OK;
}

// ---------------------------------------------------------------------------
// inputs
// ---------------------------------------------------------------------------
int mshqc_cd_set_vectors(mshqc_cd_ctx* ctx, const double* L, int64_t nbf, int64_t nvec,
                         int layout, int where) {
    CD_CHECK_CTX();
    if (nbf <= 0 || nvec <= 0) return set_error(MSHQC_CD_ERR_ARG, "nbf and nvec must be positive");
    if (!L) return set_error(MSHQC_CD_ERR_ARG, "L is null");
    if (layout != MSHQC_CD_LAYOUT_FULL && layout != MSHQC_CD_LAYOUT_PACKED)
        return set_error(MSHQC_CD_ERR_ARG, "unknown layout");
    if (where != MSHQC_CD_HOST && where != MSHQC_CD_DEVICE)
        return set_error(MSHQC_CD_ERR_ARG, "unknown pointer location");
    if (where == MSHQC_CD_DEVICE && !is_device_pointer(L))
        return set_error(MSHQC_CD_ERR_ARG, "L is not a device pointer");
    DeviceGuard g(ctx->device);
    const int64_t N = nbf, M = nvec;
    const size_t full_bytes = sizeof(double) * (size_t)M * N * N;
    ctx->invalidate_all();
    CD_ALLOC(ctx->L, full_bytes, false);
    double* dL = static_cast<double*>(ctx->L.p);
    if (layout == MSHQC_CD_LAYOUT_FULL) {
        if (where == MSHQC_CD_HOST) {
            int rc = upload(ctx, dL, L, full_bytes);
            if (rc) return rc;
        } else {
            CD_CUDA(cudaMemcpyAsync(dL, L, full_bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        }
    } else {
        const int64_t tri = N * (N + 1) / 2;
        const int64_t qchunk = std::max<int64_t>(1, std::min<int64_t>(M, (int64_t(256) << 20) / (tri * 8)));
        CD_ALLOC(ctx->scratch, sizeof(double) * (size_t)qchunk * tri, false);
        for (int64_t q0 = 0; q0 < M; q0 += qchunk) {
            const int64_t nq = std::min(qchunk, M - q0);
            const double* src = L + q0 * tri;
            const double* dsrc = src;
            if (where == MSHQC_CD_HOST) {
                int rc = upload(ctx, ctx->scratch.p, src, sizeof(double) * nq * tri);
                if (rc) return rc;
                dsrc = static_cast<const double*>(ctx->scratch.p);
            }
            unpack_vectors_kernel<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(dsrc, dL + q0 * N * N, N,
                                                                           nq);
            ctx->launches++;
            CD_CUDA(cudaGetLastError());
            if (where == MSHQC_CD_HOST) CD_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    }
    ctx->N = N;
    ctx->M = M;
    ctx->Mp = round_up(M, 16);
    ctx->L_set = true;
    ctx->L_gen = false;
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}

int mshqc_cd_set_orbitals(mshqc_cd_ctx* ctx, int spin, const double* C, const double* eps,
                          int64_t nocc, int where) {
    CD_CHECK_CTX();
    if (spin != MSHQC_CD_ALPHA && spin != MSHQC_CD_BETA)
        return set_error(MSHQC_CD_ERR_ARG, "spin must be 0 (alpha) or 1 (beta)");
    if (!C || !eps) return set_error(MSHQC_CD_ERR_ARG, "C and eps must be non-null");
    if (!ctx->L_set) return set_error(MSHQC_CD_ERR_STATE, "set_vectors must precede set_orbitals");
    const int64_t N = ctx->N;
    if (nocc < 1 || nocc >= N)
        return set_error(MSHQC_CD_ERR_ARG, "nocc must satisfy 1 <= nocc < nbf");
    DeviceGuard g(ctx->device);
    SpinState& s = ctx->spin[spin];
    CD_ALLOC(s.C, sizeof(double) * N * N, false);
    CD_ALLOC(s.eps, sizeof(double) * N, false);
    if (where == MSHQC_CD_HOST) {
        if (!host_all_finite(C, N * N)) return set_error(MSHQC_CD_ERR_NUMERIC, "C contains NaN/Inf");
        if (!host_all_finite(eps, N)) return set_error(MSHQC_CD_ERR_NUMERIC, "eps contains NaN/Inf");
        int rc = upload(ctx, s.C.p, C, sizeof(double) * N * N);
        if (rc) return rc;
        rc = upload(ctx, s.eps.p, eps, sizeof(double) * N);
        if (rc) return rc;
    } else {
        CD_CUDA(cudaMemcpyAsync(s.C.p, C, sizeof(double) * N * N, cudaMemcpyDeviceToDevice, ctx->stream));
        CD_CUDA(cudaMemcpyAsync(s.eps.p, eps, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
        int rc = check_finite_device(ctx, static_cast<double*>(s.C.p), N * N, "C");
        if (rc) return rc;
        rc = check_finite_device(ctx, static_cast<double*>(s.eps.p), N, "eps");
        if (rc) return rc;
    }
    s.nocc = nocc;
    s.set = true;
    s.invalidate();
    ctx->diag_os_valid = false;
    if (ctx->Y_spin == spin) ctx->Y_spin = -1;
    CD_CUDA(cudaStreamSynchronize(ctx->stream));
    return MSHQC_CD_OK;
}

// ---------------------------------------------------------------------------
// forward
// ---------------------------------------------------------------------------
int mshqc_cd_transform(mshqc_cd_ctx* ctx, int spin, int precision, double* B_out, int where) {
    CD_CHECK_CTX();
    if (spin != 0 && spin != 1) return set_error(MSHQC_CD_ERR_ARG, "bad spin");
    DeviceGuard g(ctx->device);
    int rc = ensure_transform(ctx, spin, precision);
    if (rc) return rc;
    if (B_out) {
        SpinState& s = ctx->spin[spin];
        const int64_t o = s.nocc, v = ctx->N - s.nocc, M = ctx->M;
        // compact [i][a][Q] copy out of the padded device layout
        for (int64_t i = 0; i < o; ++i) {
            const double* src = static_cast<const double*>(s.B64.p) + (size_t)i * s.vp * ctx->Mp;
            CD_CUDA(cudaMemcpy2DAsync(B_out + (size_t)i * v * M, sizeof(double) * M, src,
                                      sizeof(double) * ctx->Mp, sizeof(double) * M, v,
                                      where == MSHQC_CD_DEVICE ? cudaMemcpyDeviceToDevice
                                                               : cudaMemcpyDeviceToHost,
                                      ctx->stream));
        }
        CD_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return MSHQC_CD_OK;
}

int mshqc_cd_mp2_energy(mshqc_cd_ctx* ctx, int kind, int precision, mshqc_cd_energy* out) {
    CD_CHECK_CTX();
    if (!out) return set_error(MSHQC_CD_ERR_ARG, "out is null");
    if (kind != MSHQC_CD_RESTRICTED && kind != MSHQC_CD_UNRESTRICTED)
        return set_error(MSHQC_CD_ERR_ARG, "unknown kind");
    if (precision != MSHQC_CD_FP64 && precision != MSHQC_CD_FP16X3)
        return set_error(MSHQC_CD_ERR_ARG, "unknown precision");
    DeviceGuard g(ctx->device);
    return run_energy(ctx, kind, precision, out);
}

int mshqc_cd_pair_energies(mshqc_cd_ctx* ctx, int block, double* out, int where) {
    CD_CHECK_CTX();
    if (!out) return set_error(MSHQC_CD_ERR_ARG, "out is null");
    if (block < 0 || block > 2) return set_error(MSHQC_CD_ERR_ARG, "block must be 0, 1 or 2");
    const auto& pe = ctx->pair_energy[block];
    if (pe.empty()) return set_error(MSHQC_CD_ERR_STATE, "no pair energies for this block yet");
    if (where == MSHQC_CD_DEVICE) {
        DeviceGuard g(ctx->device);
        CD_CUDA(cudaMemcpy(out, pe.data(), pe.size() * sizeof(double), cudaMemcpyHostToDevice));
    } else {
        std::memcpy(out, pe.data(), pe.size() * sizeof(double));
    }
    return MSHQC_CD_OK;
}

int mshqc_cd_mp2_gradient(mshqc_cd_ctx* ctx, int kind, int precision, mshqc_cd_energy* e_out,
                          double* dC_a, double* dC_b, double* deps_a, double* deps_b, int where) {
    CD_CHECK_CTX();
    if (kind != MSHQC_CD_RESTRICTED && kind != MSHQC_CD_UNRESTRICTED)
        return set_error(MSHQC_CD_ERR_ARG, "unknown kind");
    if (precision != MSHQC_CD_FP64 && precision != MSHQC_CD_FP16X3)
        return set_error(MSHQC_CD_ERR_ARG, "unknown precision");
    DeviceGuard g(ctx->device);
    return run_gradient(ctx, kind, precision, e_out, dC_a, dC_b, deps_a, deps_b, where);
}

}  // extern "C"
