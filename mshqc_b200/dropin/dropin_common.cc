// Process-wide device context and error conversion of the drop-in build.
#include "dropin_common.h"

#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>

namespace mshqc_dropin {

namespace {
struct Holder {
    mshqc_cd_ctx* ctx = nullptr;
    ~Holder() {
        if (ctx) mshqc_cd_ctx_destroy(ctx);
    }
};
Holder g_holder;
std::mutex g_mutex;
}  // namespace

void check(int rc) {
    if (rc != MSHQC_CD_OK) throw std::runtime_error(std::string("libmshqc_cuda: ") + mshqc_cd_last_error());
}

mshqc_cd_ctx* context() {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_holder.ctx) {
        const char* env = std::getenv("MSHQC_DEVICE");
        check(mshqc_cd_ctx_create(env ? std::atoi(env) : 0, &g_holder.ctx));
    }
    return g_holder.ctx;
}

int precision() {
    const char* env = std::getenv("MSHQC_CD_PRECISION");
    return (env && std::strcmp(env, "fp16x3") == 0) ? MSHQC_CD_FP16X3 : MSHQC_CD_FP64;
}

size_t t2_max_bytes() {
    const char* env = std::getenv("MSHQC_T2_MAX_BYTES");
    return env ? (size_t)std::strtoull(env, nullptr, 10) : (size_t(8) << 30);
}

}  // namespace mshqc_dropin
