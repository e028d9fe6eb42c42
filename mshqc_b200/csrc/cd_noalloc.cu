// mshqc_cd_rmp2_energy_noalloc: the FP64 closed-shell pair-energy pass on
// caller-owned device buffers, with every piece of scratch in one file-scope
// device array, so the call allocates nothing.
//
// Scratch (g_noalloc_scratch, kNoallocScratchBytes), rebuilt in stream order
// by every call before it is read, so none of it needs to start at zero:
//   [pairs int2 * npairs][blocks int2 * nblocks]   (256-byte aligned end)
//   [partial double * units][partial2 double * units][pair_sum double * 2 npairs]
// units = npairs * nblocks, npairs = o (o + 1) / 2, nblocks = nb (nb + 1) / 2,
// nb = vp / 64.
//
// All calls on one device share the array: two calls that overlap in time
// (different streams, or different host threads without ordering) race on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "cd_common.cuh"
#include "cd_internal.h"
#include "pair_energy_f64.cuh"

namespace mshqc_cd {
namespace {

constexpr size_t kNoallocScratchBytes = MSHQC_CD_NOALLOC_SCRATCH_BYTES;
static_assert(kNoallocScratchBytes % 256 == 0, "scratch size must be a multiple of 256 bytes");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_setup_ctx[kMaxDevices] = {};   // context of the cached set-up (0: none)

// Unique id of the calling thread's current CUDA context (never reused within
// a process, so a context made after cudaDeviceReset has a new one), through
// the driver entry points the runtime hands out; 0 when unavailable.
unsigned long long current_context_id() {
    using GetCurrentFn = int (*)(void**);
    using GetIdFn = int (*)(void*, unsigned long long*);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1{}, q2{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrentFn>(f1);
            get_id = reinterpret_cast<GetIdFn>(f2);
        }
        looked_up = true;
    }
    if (!get_current || !get_id) return 0;
    void* c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != 0 || !c || get_id(c, &id) != 0) return 0;
    return id;
}

// (i, j), i <= j, row by row; and (x, y), x <= y, row by row -- the unit order
// of the context path's tables.
static __global__ void noalloc_tables_kernel(int o, int nb, int2* __restrict__ pairs, int2* __restrict__ blocks) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t np2 = (int64_t)o * o, nb2 = (int64_t)nb * nb;
    if (t < np2) {
        const int i = (int)(t / o), j = (int)(t % o);
        if (j >= i) pairs[(int64_t)i * o - (int64_t)i * (i - 1) / 2 + (j - i)] = make_int2(i, j);
    } else if (t < np2 + nb2) {
        const int64_t u = t - np2;
        const int x = (int)(u / nb), y = (int)(u % nb);
        if (y >= x) blocks[(int64_t)x * nb - (int64_t)x * (x - 1) / 2 + (y - x)] = make_int2(x, y);
    }
}

// Once per device and CUDA context, with that device current: the address of
// the scratch array and the kernel's shared-memory limit.  Both belong to the
// context, so a new context on the device (after cudaDeviceReset) sets up
// again; without the context id the set-up runs on every call (it allocates
// nothing either way).
int noalloc_setup(int dev, void** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx_id = current_context_id();
    if (g_scratch_ptr[dev] && ctx_id != 0 && g_setup_ctx[dev] == ctx_id) {
        *out = g_scratch_ptr[dev];
        return MSHQC_CD_OK;
    }
    int major = 0, minor = 0;
    cudaError_t e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (e != cudaSuccess) return cuda_error(e, "device query");
    if (major != 10)
        return set_error(MSHQC_CD_ERR_UNSUPPORTED, "device " + std::to_string(dev) + " is sm_" +
                                                       std::to_string(major * 10 + minor) +
                                                       "; this library is built for sm_100a");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(scratch)");
    e = cudaFuncSetAttribute(pair_energy_f64_kernel<PAIR_RESTRICTED>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)pair_f64_detail::SMEM_BYTES);
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute(pair kernel)");
    g_scratch_ptr[dev] = p;
    g_setup_ctx[dev] = ctx_id;
    *out = p;
    return MSHQC_CD_OK;
}

}  // namespace
}  // namespace mshqc_cd

using namespace mshqc_cd;

extern "C" MSHQC_CD_API int mshqc_cd_rmp2_energy_noalloc(const double* B, const double* eps, int64_t nocc,
                                                         int64_t nvir, int64_t nvec, double* energy,
                                                         void* stream) {
    if (!B || !eps || !energy) return set_error(MSHQC_CD_ERR_ARG, "B, eps and energy must be device pointers");
    if (nocc < 1 || nvir < 1 || nvec < 1)
        return set_error(MSHQC_CD_ERR_ARG, "nocc, nvir and nvec must be positive");
    const int64_t vp = round_up(nvir, 64), Mp = round_up(nvec, 16), nb = vp / 64;
    if (nocc > (1 << 20) || vp > (1 << 20) || Mp > (int64_t(1) << 30))
        return set_error(MSHQC_CD_ERR_ARG, "nocc, nvir or nvec out of range");
    const int64_t npairs = nocc * (nocc + 1) / 2, nblocks = nb * (nb + 1) / 2;
    const int64_t units = npairs * nblocks;
    const int64_t table_bytes = round_up(8 * (npairs + nblocks), 256);
    const int64_t need = table_bytes + 16 * units + 16 * npairs;
    if (need > (int64_t)kNoallocScratchBytes || units > INT32_MAX)
        return set_error(MSHQC_CD_ERR_ARG,
                         "scratch of " + std::to_string(need) + " bytes needed (nocc=" + std::to_string(nocc) +
                             ", nvir=" + std::to_string(nvir) + "); the static scratch holds " +
                             std::to_string(kNoallocScratchBytes) +
                             " bytes: use mshqc_cd_mp2_energy for this size");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_error(MSHQC_CD_ERR_UNSUPPORTED, "device index out of range");
    void* scratch = nullptr;
    const int rc = noalloc_setup(dev, &scratch);
    if (rc != MSHQC_CD_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    unsigned char* base = static_cast<unsigned char*>(scratch);
    int2* pairs = reinterpret_cast<int2*>(base);
    int2* blocks = pairs + npairs;
    double* partial = reinterpret_cast<double*>(base + table_bytes);
    double* partial2 = partial + units;
    double* pair_sum = partial2 + units;

    const int64_t tt = nocc * nocc + nb * nb;
    noalloc_tables_kernel<<<(unsigned)cdiv(tt, 256), 256, 0, st>>>((int)nocc, (int)nb, pairs, blocks);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "table kernel launch");

    PairF64Args a{};
    a.X = B;  a.Y = B;
    a.vx = a.vy = (int)nvir;
    a.vpx = a.vpy = (int)vp;
    a.Mp = (int)Mp;
    a.eox = eps;  a.evx = eps + nocc;
    a.eoy = a.eox;  a.evy = a.evx;
    a.pairs = pairs;  a.blocks = blocks;
    a.nblocks = (int)nblocks;
    a.partial = partial;  a.partial2 = partial2;
    pair_energy_f64_kernel<PAIR_RESTRICTED>
        <<<(unsigned)units, 256, pair_f64_detail::SMEM_BYTES, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "pair kernel launch");
    // deterministic reductions straight into the caller's two doubles
    reduce_pairs_kernel<<<(unsigned)cdiv(npairs, 128), 128, 0, st>>>(partial, (int)npairs, (int)nblocks, pair_sum);
    reduce_pairs_kernel<<<(unsigned)cdiv(npairs, 128), 128, 0, st>>>(partial2, (int)npairs, (int)nblocks,
                                                                     pair_sum + npairs);
    reduce_total_kernel<<<1, 256, 0, st>>>(pair_sum, (int)npairs, energy);
    reduce_total_kernel<<<1, 256, 0, st>>>(pair_sum + npairs, (int)npairs, energy + 1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "reduction launch");
    return MSHQC_CD_OK;
}
